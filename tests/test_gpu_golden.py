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
    # against the reference of the same CT: glst_force<double> is FP64
    # throughout; glst_force<float> carries its own ~1e-6 float error, which
    # the same bars still cover
    rep = oracle.error_report(got, (d["fx"], d["fy"], d["fz"], d["en"]))
    print(case, ct, rep)
    assert rep["force_rms_rel"] <= FORCE_RMS_TOL, rep
    assert rep["energy_rel"] <= ENERGY_TOL, rep


def test_water333k_matches_reference_subset(pkg):
    """water333k: 333,333 waters (999,999 atoms), L = 215.3 A.  The fixture
    holds the reference's outputs on a seeded subset of 20,000 atoms, its
    total energy, and a digest of its full cell assignment."""
    import hashlib
    import os
    d, (x, y, z, q), box = load_case("water333k", "double")
    dev = [torch.tensor(a, dtype=torch.float64, device="cuda:0") for a in (x, y, z, q)]
    with pkg.GlstForce(len(x), float(d["tol"]), *box, rcut=float(d["rcut"])) as f:
        assert f.info().num_nodes == int(d["K"])
        f.calc_ener_force(*dev)
        fx, fy, fz, en = f.get_ef()
        e = f.energy()
        sidx, cnt, pnt = f.assignment()
    digest = hashlib.sha256(b"".join(np.ascontiguousarray(a, dtype="<u4").tobytes()
                                     for a in (sidx, cnt, pnt))).hexdigest()
    assert digest == str(d["assignment_sha256"])
    sel = d["subset"]
    dF2 = np.sum((fx[sel] - d["fx"]) ** 2 + (fy[sel] - d["fy"]) ** 2 + (fz[sel] - d["fz"]) ** 2)
    F2 = np.sum(d["fx"] ** 2 + d["fy"] ** 2 + d["fz"] ** 2)
    rel = float(np.sqrt(dF2 / F2))
    e_rel = abs(e - float(d["energy_total"])) / abs(float(d["energy_total"]))
    print("water333k force_rms_rel(subset) %.3e energy_rel %.3e" % (rel, e_rel))
    assert rel <= FORCE_RMS_TOL
    assert e_rel <= ENERGY_TOL


def test_water10k_next_order_matches_reference(pkg):
    """water10k at the next higher cubature order (tol/10: t = 101, 83, 57,
    K = 192,478 nodes) against the reference's glst_force<double>."""
    d, (x, y, z, q), box = load_case("water10k_next", "double")
    dev = [torch.tensor(a, dtype=torch.float64, device="cuda:0") for a in (x, y, z, q)]
    with pkg.GlstForce(len(x), float(d["tol"]), *box, rcut=float(d["rcut"])) as f:
        assert f.info().num_nodes == int(d["K"])
        f.calc_ener_force(*dev)
        got = f.get_ef()
        sidx, cnt, pnt = f.assignment()
    assert np.array_equal(sidx, d["sorted_idx"])
    rep = oracle.error_report(got, (d["fx"], d["fy"], d["fz"], d["en"]))
    print("water10k_next", rep)
    assert rep["force_rms_rel"] <= FORCE_RMS_TOL, rep
    assert rep["energy_rel"] <= ENERGY_TOL, rep
