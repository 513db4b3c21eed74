"""Pin the oracle to the reference (CPU).

tests/golden/*.npz hold outputs of the UNMODIFIED reference library
(glst_force<double> and glst_force<float>, built for sm_100a by oracle/Makefile
and run on a B200 by tests/golden/make_golden.py) on seeded water boxes.  The
FP64 oracle must reproduce the reference's double path to round-off and its
cell assignment bit for bit, for both calculation types.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle, planner

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def load_case(name, ct):
    d = np.load(os.path.join(GOLDEN, "%s_%s.npz" % (name, ct)))
    from glst_b200 import systems
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    x, y, z, q = systems.water_box(int(d["n_mol"]), float(d["box"]), seed=int(d["seed"]))
    assert mg.input_sha256(x, y, z, q) == str(d["input_sha256"]), "inputs differ from the fixture's"
    L = float(d["box"])
    return d, (x, y, z, q), (L, L, L)


SMALL = ["water216", "w1000_tol1e-4", "w2000_tol1e-5"]


def test_fixtures_present():
    names = {os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    for c in SMALL + ["water10k"]:
        for ct in ("double", "float"):
            assert "%s_%s.npz" % (c, ct) in names
    assert "water333k_double.npz" in names
    assert "water10k_next_double.npz" in names


@pytest.mark.parametrize("case", SMALL)
def test_oracle_reproduces_reference_double_path(store, case):
    d, (x, y, z, q), box = load_case(case, "double")
    p = planner.make_plan(len(x), float(d["tol"]), box, float(d["rcut"]), store)
    assert p.K == int(d["K"]) and p.n == tuple(int(v) for v in d["ncell"])
    got = oracle.glst(x, y, z, q, p)
    rep = oracle.error_report(got, (d["fx"], d["fy"], d["fz"], d["en"]))
    assert rep["force_rms_rel"] < 1e-13, rep
    assert rep["energy_rel"] < 1e-13, rep


@pytest.mark.slow
@pytest.mark.parametrize("case", ["water10k", "water10k_next"])
def test_oracle_reproduces_reference_double_path_large(store, case):
    """10,000 waters at the default order (K = 100,532) and the next order
    (tol / 10, K = 192,478): a full FP64 solve each, ~20-40 s on 8 cores."""
    d, (x, y, z, q), box = load_case(case, "double")
    p = planner.make_plan(len(x), float(d["tol"]), box, float(d["rcut"]), store)
    assert p.K == int(d["K"]) and p.n == tuple(int(v) for v in d["ncell"])
    got = oracle.glst(x, y, z, q, p)
    rep = oracle.error_report(got, (d["fx"], d["fy"], d["fz"], d["en"]))
    assert rep["force_rms_rel"] < 1e-13, rep
    assert rep["energy_rel"] < 1e-13, rep


@pytest.mark.parametrize("case", SMALL + ["water10k"])
@pytest.mark.parametrize("ct", ["double", "float"])
def test_oracle_assignment_bitexact_with_reference(store, case, ct):
    d, (x, y, z, q), box = load_case(case, ct)
    n, l = planner.cell_grid(box, float(d["rcut"]), ct)
    assert n == tuple(int(v) for v in d["ncell"])
    p = planner.Plan()
    p.n, p.cell_dim, p.ncell, p.ct = n, l, n[0] * n[1] * n[2], ct
    p.kx = p.ky = p.kz = p.w = np.zeros(0)
    p.group = np.zeros(0, dtype=np.uint32)
    p.K, p.ngroup, p.has_far = 0, 0, False
    p.groups = {"r_in": [], "r_out": []}
    _ac, cnt, pnt, sidx = oracle.assign(x, y, z, p)
    assert np.array_equal(cnt, d["cell_count"])
    assert np.array_equal(pnt, d["cell_point"])
    assert np.array_equal(sidx, d["sorted_idx"])


@pytest.mark.parametrize("case", SMALL)
def test_reference_float_path_error_is_bounded(store, case):
    """The reference's own float path, against FP64: the error budget a float
    user of the reference already accepts (recorded, and bounded loosely)."""
    d, (x, y, z, q), box = load_case(case, "float")
    p = planner.make_plan(len(x), float(d["tol"]), box, float(d["rcut"]), store)
    ref64 = oracle.glst(x, y, z, q, p)
    rep = oracle.error_report((d["fx"], d["fy"], d["fz"], d["en"]), ref64)
    assert rep["force_rms_rel"] < 1e-4 and rep["energy_rel"] < 1e-6, rep
