"""The CUDA path against the UNMODIFIED reference's own outputs (GPU).

For every golden case (tests/golden/, made by the reference library on a
B200), the engine -- called through the C-ABI -- must give
  * the reference's cell assignment bit for bit (sorted_idx, counts, offsets),
  * forces within 1e-5 relative RMS and total energy within 1e-7 relative
    of the reference's glst_force<double> outputs.
Its float-CT mode is also checked against glst_force<float>'s assignment.
"""
import numpy as np
import pytest

from oracle import oracle
from test_golden import load_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FORCE_RMS_TOL = 1e-5
ENERGY_TOL = 1e-7


@pytest.mark.parametrize("case", ["water216", "w1000_tol1e-4", "w2000_tol1e-5", "water10k"])
@pytest.mark.parametrize("ct", ["double", "float"])
def test_cuda_path_matches_reference(pkg, case, ct):
    d, (x, y, z, q), box = load_case(case, ct)
    dev = [torch.tensor(a, dtype=torch.float64, device="cuda:0") for a in (x, y, z, q)]
    with pkg.GlstForce(len(x), float(d["tol"]), *box, rcut=float(d["rcut"]), ct=ct) as f:
        assert f.info().num_nodes == int(d["K"])
        f.calc_ener_force(*dev)
        got = f.get_ef()
        f.check()
        sidx, cnt, pnt = f.assignment()
    assert np.array_equal(sidx, d["sorted_idx"])
    assert np.array_equal(cnt, d["cell_count"])
    assert np.array_equal(pnt, d["cell_point"])
    if ct == "double":
        rep = oracle.error_report(got, (d["fx"], d["fy"], d["fz"], d["en"]))
        print(case, ct, rep)
        assert rep["force_rms_rel"] <= FORCE_RMS_TOL, rep
        assert rep["energy_rel"] <= ENERGY_TOL, rep
