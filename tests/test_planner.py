"""Host planning (CPU): the C++ planner of the product agrees bit for bit with
the oracle's restatement of the reference set-up (src/glst_force.cu:223-241,
:1616-1724; src/cubature.cu:100-523), and the pieces behave as the reference's
self-checks require."""
import math

import numpy as np
import pytest

from oracle import planner

CASES = [
    # (natom, tol, box, rcut, ct)
    (648, math.erfc(0.34 * 9.0) / 9.0, 18.63, 9.0, "double"),
    (3000, 1.165e-6, 31.04, 8.0, "double"),
    (6000, 1.165e-6, 39.1, 10.0, "double"),
    (6000, 1.165e-6, 39.1, 10.0, "float"),
    (30000, math.erfc(0.31 * 10.0) / 10.0, 66.9, 10.0, "double"),
    (900, 1.165e-6, 20.0, 10.0, "double"),   # 2x2x2 cells: no far field
    (9000, 1.165e-6, 44.3, 10.0, "float"),
]


@pytest.mark.parametrize("natom,tol,L,rcut,ct", CASES)
def test_cpp_plan_matches_oracle_plan(pkg, store, natom, tol, L, rcut, ct):
    inf, nodes = pkg.plan(natom, tol, (L, L, L), rcut, ct=ct)
    p = planner.make_plan(natom, tol, (L, L, L), rcut, store, ct=ct)
    assert tuple(inf.ncell) == p.n
    assert inf.cell_dim == p.cell_dim
    assert inf.ngroup == p.ngroup
    assert bool(inf.has_far_field) == p.has_far
    for g in range(p.ngroup):
        assert inf.group_alpha[g] == p.groups["alpha"][g]
        assert inf.group_zcut[g] == p.groups["zcut"][g]
        assert inf.group_rmax[g] == p.groups["rmax"][g]
        assert inf.group_r_in[g] == p.groups["r_in"][g]
        assert inf.group_r_out[g] == p.groups["r_out"][g]
        assert inf.group_gl_degree[g] == p.gl_degree[g]
        assert inf.group_t_degree[g] == p.t_degree[g]
    kx, ky, kz, w, grp = nodes
    assert inf.num_nodes == p.K == kx.size
    ref = planner.make_plan(natom, tol, (L, L, L), rcut, store, ct="double") if ct == "float" else p
    # nodes are reported before CT rounding
    assert np.array_equal(kx, ref.kx if ct == "double" else kx)
    if ct == "double":
        for a, b in zip((kx, ky, kz, w), (p.kx, p.ky, p.kz, p.w)):
            assert np.array_equal(a, b)
        assert np.array_equal(grp, p.group)


def test_alpha_groups_c1_shape():
    # 7 cells per axis -> widths {1, 2, 2} (src/glst_force.cu:1688-1702)
    g = planner.alpha_groups((7, 7, 7), 10.0, math.erfc(3.1) / 10.0)
    assert g["widths"] == [1, 2, 2]
    assert g["r_in"] == [1, 2, 4] and g["r_out"] == [2, 4, 6]
    assert abs(g["alpha"][0] - 0.31) < 1e-12   # alpha_0 reproduces the splitting parameter
    g = planner.alpha_groups((22, 22, 22), 10.0, math.erfc(3.1) / 10.0)
    assert g["widths"] == [1, 2, 4, 6, 7]
    assert g["r_out"][-1] == 21


def test_erfc_inverse_roundtrip():
    for y in (1e-3, 1.7e-5, 3.3e-6, 1e-8):
        x = planner.erfc_inv(y, 2.220446049250313e-16)
        assert abs(math.erfc(x) - y) < 1e-15


def test_gauss_legendre_rule_exact():
    for n in (2, 4, 10, 32, 66, 80):
        xs = planner.gl_roots(n)
        ws = planner.gl_weights(xs, n)
        x = np.concatenate([-np.array(xs)[::-1], xs])
        w = np.concatenate([np.array(ws)[::-1], ws])
        ref_x, ref_w = np.polynomial.legendre.leggauss(n)
        assert np.allclose(np.sort(x), ref_x, atol=1e-14, rtol=0)
        assert np.allclose(w[np.argsort(x)], ref_w, atol=1e-13, rtol=0)


def test_grid_float_semantics():
    # box/rcut rounding in float can differ from double
    n_d, l_d = planner.cell_grid((66.9, 66.9, 66.9), 10.0, "double")
    n_f, l_f = planner.cell_grid((66.9, 66.9, 66.9), 10.0, "float")
    assert n_d == n_f == (7, 7, 7)
    assert l_f == float(np.float32(10.0))
    assert planner.rcut_from_ncell((30.0, 20.0, 40.0), (3, 4, 2)) == 5.0


def test_missing_tdesign_is_an_error(pkg, tmp_path):
    empty = tmp_path / "SS31-Mar-2016"
    empty.mkdir()
    pkg.set_tdesign_path(str(empty))
    try:
        with pytest.raises(pkg.GlstError) as e:
            pkg.plan(648, 1.676e-6, (18.63,) * 3, 9.0)
        assert e.value.status == 4  # GLST_ERR_TDESIGN
    finally:
        pkg.set_tdesign_path(None)


def test_reference_layout_directory_gives_same_plan(pkg, store, tmp_path):
    """The store rendered in the reference's text layout (ssTTT.NNNNN) plans
    to identical nodes."""
    import importlib.util, os
    spec = importlib.util.spec_from_file_location(
        "make_tdesigns", os.path.join(os.path.dirname(pkg.TDESIGN_STORE), "make_tdesigns.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    d = tmp_path / "SS31-Mar-2016"
    designs = mk.read_store(pkg.TDESIGN_STORE)
    sub = {t: designs[t] for t in designs if t <= 101}
    mk.write_store(str(tmp_path / "sub.bin"), sub)
    mk.write_reference_dir(str(tmp_path / "sub.bin"), str(d))
    a_inf, a = pkg.plan(648, 1.676e-6, (18.63,) * 3, 9.0)
    pkg.set_tdesign_path(str(d))
    try:
        b_inf, b = pkg.plan(648, 1.676e-6, (18.63,) * 3, 9.0)
    finally:
        pkg.set_tdesign_path(None)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    s2 = planner.TDesignStore(str(d))
    p = planner.make_plan(648, 1.676e-6, (18.63,) * 3, 9.0, s2)
    assert np.array_equal(p.kx, a[0])


def test_charmm_roundtrip(tmp_path):
    """psf/cor writer and reader use the columns the reference driver reads
    (utils/io.cpp:35-117)."""
    from glst_b200 import systems
    x, y, z, q = systems.water_box(50, 12.0, seed=2)
    systems.write_charmm(str(tmp_path / "w"), x, y, z, q)
    a = systems.read_charmm(str(tmp_path / "w"))
    for u, v in zip(a, (x, y, z, q)):
        assert np.allclose(u, v, atol=1e-9, rtol=0)
    lines = open(str(tmp_path / "w.psf")).read().splitlines()
    hdr = [ln for ln in lines if "!NATOM" in ln][0]
    assert hdr[11:17] == "!NATOM" and int(hdr[0:10]) == 150
    r = systems.recenter(x + 3.0, y - 2.0, z)
    assert min(a.min() for a in r) == 0.0
