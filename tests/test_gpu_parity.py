"""GPU parity: the CUDA path (called through the C-ABI) against the FP64 oracle.

Bars (stated here, checked below):
  * cell assignment (sorted_idx, cell counts, offsets): bit-exact;
  * forces: relative RMS error sqrt(sum|dF|^2 / sum|F|^2) <= 1e-5;
  * total energy 0.5*sum(en): relative error <= 1e-7;
  * the same call twice gives bit-identical results (fixed-order reductions).
"""
import math

import numpy as np
import pytest

from oracle import oracle, planner

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5
ENERGY_TOL = 1e-7

torch = pytest.importorskip("torch")


def _dev(a):
    return torch.tensor(np.asarray(a), dtype=torch.float64, device="cuda:0")


def _water(n_mol, L, seed):
    from glst_b200 import systems
    return systems.water_box(n_mol, L, seed=seed)


_ORACLE_CACHE = {}


def _oracle(key, x, y, z, q, tol, L, rcut, store, ct="double"):
    if key not in _ORACLE_CACHE:
        p = planner.make_plan(len(x), tol, (L, L, L), rcut, store, ct=ct)
        _ORACLE_CACHE[key] = (p, oracle.glst(x, y, z, q, p))
    return _ORACLE_CACHE[key]


def _run(pkg, x, y, z, q, tol, L, rcut, ct="double"):
    f = pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut, ct=ct)
    f.calc_ener_force(_dev(x), _dev(y), _dev(z), _dev(q))
    out = f.get_ef()
    return f, out


SYSTEMS = {
    # name: (molecules, box, rcut, tol, seed)
    "w1000_tol1e-4": (1000, 31.04, 8.0, 1e-4, 3),
    "w500_tol1e-5": (500, 24.6, 6.0, 1e-5, 4),
    "w2000_tol1e-5": (2000, 39.1, 10.0, 1e-5, 5),
    "w1000_c1tol": (1000, 31.04, 8.0, 1.165e-6, 6),
}


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_far_field_parity(pkg, store, name):
    n_mol, L, rcut, tol, seed = SYSTEMS[name]
    x, y, z, q = _water(n_mol, L, seed)
    f, got = _run(pkg, x, y, z, q, tol, L, rcut)
    f.check()
    p, ref = _oracle(name, x, y, z, q, tol, L, rcut, store)
    assert f.info().num_nodes == p.K and p.has_far
    rep = oracle.error_report(got, ref)
    assert rep["force_rms_rel"] <= FORCE_RMS_TOL, rep
    assert rep["energy_rel"] <= ENERGY_TOL, rep
    # the engine's device-side total equals 0.5 * sum(en)
    assert abs(f.energy() - 0.5 * np.sum(got[3])) <= 1e-12 * abs(f.energy())
    # assignment bit-exact with the reference semantics
    _ac, cnt, pnt, sidx = oracle.assign(x, y, z, p)
    g_sidx, g_cnt, g_pnt = f.assignment()
    assert np.array_equal(g_cnt, cnt) and np.array_equal(g_pnt, pnt) and np.array_equal(g_sidx, sidx)
    f.close()


def test_water216_matches_direct_coulomb(pkg, store):
    """water216: 216 waters, L = 18.63 A, rcut 9, alpha 0.34.  All atoms sit
    in cells 0..1 of the 3x3x3 grid, so the far field is empty and GLST equals
    the direct sum."""
    from glst_b200 import systems
    s = systems.config_system("water216", seed=0)
    L = s["box"][0]
    f, got = _run(pkg, s["x"], s["y"], s["z"], s["q"], s["tol"], L, s["rcut"])
    ref = oracle.coulomb(s["x"], s["y"], s["z"], s["q"])
    rep = oracle.error_report(got, ref)
    assert rep["force_rms_rel"] <= 1e-12 and rep["energy_rel"] <= 1e-12, rep
    f.close()


def test_determinism_bitwise(pkg):
    n_mol, L, rcut, tol, seed = SYSTEMS["w1000_tol1e-4"]
    x, y, z, q = _water(n_mol, L, seed)
    f = pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut)
    d = [_dev(a) for a in (x, y, z, q)]
    f.calc_ener_force(*d)
    a = f.get_ef()
    e1 = f.energy()
    f.calc_ener_force(*d)
    b = f.get_ef()
    assert all(np.array_equal(u, v) for u, v in zip(a, b))
    assert e1 == f.energy()
    f.close()


def test_phase_api_equals_fused_call(pkg):
    n_mol, L, rcut, tol, seed = SYSTEMS["w1000_tol1e-4"]
    x, y, z, q = _water(n_mol, L, seed)
    d = [_dev(a) for a in (x, y, z, q)]
    f = pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut)
    f.calc_ener_force(*d)
    a = f.get_ef()
    f.assign_atoms(*d)
    f.calc_sf()
    f.sum_rmt_sf()
    f.calc_lr_ef()
    f.calc_sr_ef()
    f.comm_ef()
    b = f.get_ef()
    assert all(np.array_equal(u, v) for u, v in zip(a, b))
    # cell-ordered outputs (the reference's fx()...en()) are the input-order
    # outputs permuted by sorted_idx
    sidx, _, _ = f.assignment()
    for dptr, host in zip(f.cell_outputs(), b):
        cell = _copy_device_doubles(dptr, len(x))
        assert np.array_equal(cell, host[sidx])
    f.close()


def _copy_device_doubles(dptr, n):
    import ctypes
    import glob
    import os
    libs = glob.glob(os.path.join(os.path.dirname(torch.__file__), "lib", "libcudart*.so*"))
    libs += glob.glob("/usr/local/cuda/lib64/libcudart.so*")
    rt = ctypes.CDLL(libs[0])
    out = np.empty(n)
    torch.cuda.synchronize()
    assert rt.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(dptr), ctypes.c_size_t(8 * n), 2) == 0
    return out


def test_host_path_equals_device_path(pkg):
    n_mol, L, rcut, tol, seed = SYSTEMS["w500_tol1e-5"]
    x, y, z, q = _water(n_mol, L, seed)
    f = pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut)
    a = f.compute_host(x, y, z, q)
    f.calc_ener_force(*[_dev(v) for v in (x, y, z, q)])
    b = f.get_ef()
    assert all(np.array_equal(u, v) for u, v in zip(a, b))
    # device-side get_ef into caller tensors
    outs = [torch.empty(len(x), dtype=torch.float64, device="cuda:0") for _ in range(4)]
    f.get_ef(*outs)
    torch.cuda.synchronize()
    assert all(np.array_equal(o.cpu().numpy(), v) for o, v in zip(outs, b))
    f.close()


def test_float_ct_assignment_bitexact(pkg, store):
    """glst_force<float> semantics: grid and binning in float.  Atoms placed
    exactly on and next to cell faces, where float and double binning can
    disagree."""
    rng = np.random.default_rng(11)
    L, rcut, tol = 40.0, 10.0, 1e-4
    n = 3000
    pts = rng.uniform(0.0, L, size=(n, 3))
    faces = np.array([0.0, 10.0, 20.0, 30.0, 40.0])
    k = n // 3
    pts[:k, 0] = rng.choice(faces, k) + rng.choice([-1, 0, 1], k) * np.spacing(20.0)
    pts[:k, 1] = rng.choice(faces, k) * (1 + 1e-8 * rng.choice([-1, 0, 1], k))
    q = rng.choice([-0.8, 0.4], n)
    x, y, z = (np.ascontiguousarray(pts[:, i]) for i in range(3))
    for ct in ("float", "double"):
        f = pkg.GlstForce(n, tol, L, L, L, rcut=rcut, ct=ct)
        f.calc_ener_force(*[_dev(v) for v in (x, y, z, q)])
        p = planner.make_plan(n, tol, (L, L, L), rcut, store, ct=ct)
        _ac, cnt, pnt, sidx = oracle.assign(x, y, z, p)
        g_sidx, g_cnt, g_pnt = f.assignment()
        assert np.array_equal(g_cnt, cnt), ct
        assert np.array_equal(g_sidx, sidx), ct
        f.close()


def test_pure_near_field_grid(pkg):
    """<= 2 cells on an axis: no far field (src/glst_force.cu:667-670); the
    result is the direct sum over the 27-cell neighbourhood, which for a
    2x2x2 grid is every pair."""
    x, y, z, q = _water(300, 19.5, 7)
    f, got = _run(pkg, x, y, z, q, 1e-5, 19.5, 10.0)
    assert f.info().has_far_field == 0
    ref = oracle.coulomb(x, y, z, q)
    rep = oracle.error_report(got, ref)
    assert rep["force_rms_rel"] <= 1e-12 and rep["energy_rel"] <= 1e-12, rep
    f.close()


def test_edge_sizes(pkg):
    # no atoms
    f = pkg.GlstForce(0, 1e-4, 40.0, 40.0, 40.0, rcut=10.0)
    e = torch.empty(0, dtype=torch.float64, device="cuda:0")
    f.calc_ener_force(e, e, e, e)
    assert f.energy() == 0.0
    f.close()
    # one atom: no interactions
    f = pkg.GlstForce(1, 1e-4, 40.0, 40.0, 40.0, rcut=10.0)
    one = [_dev([v]) for v in (5.0, 5.0, 5.0, 1.0)]
    f.calc_ener_force(*one)
    fx, fy, fz, en = f.get_ef()
    assert fx[0] == 0.0 and en[0] == 0.0
    f.close()
    # two atoms in far-apart cells: far field only, close to 1/r
    f = pkg.GlstForce(2, 1e-6, 40.0, 40.0, 40.0, rcut=10.0)
    pts = [_dev(v) for v in ([2.0, 38.0], [3.0, 37.0], [4.0, 36.0], [1.0, -1.0])]
    f.calc_ener_force(*pts)
    fx, fy, fz, en = f.get_ef()
    r = math.sqrt(36.0 ** 2 + 34.0 ** 2 + 32.0 ** 2)
    assert abs(en[0] - (-1.0 / r)) < 1e-5
    f.close()


def test_atoms_outside_box_are_clamped(pkg, store):
    rng = np.random.default_rng(5)
    n, L = 2000, 40.0
    pts = rng.uniform(-3.0, L + 3.0, size=(n, 3))
    q = rng.choice([-0.5, 0.5], n)
    x, y, z = (np.ascontiguousarray(pts[:, i]) for i in range(3))
    f, got = _run(pkg, x, y, z, q, 1e-4, L, 10.0)
    p, ref = _oracle("outside", x, y, z, q, 1e-4, L, 10.0, store)
    _ac, cnt, pnt, sidx = oracle.assign(x, y, z, p)
    g_sidx, g_cnt, _ = f.assignment()
    assert np.array_equal(g_sidx, sidx) and np.array_equal(g_cnt, cnt)
    rep = oracle.error_report(got, ref)
    assert rep["force_rms_rel"] <= FORCE_RMS_TOL, rep
    f.close()


@pytest.mark.slow
def test_water10k_parity(pkg, store):
    """water10k workload: 10,000 waters, L = 66.9 A, rcut 10, alpha 0.31."""
    from glst_b200 import systems
    s = systems.config_system("water10k", seed=0)
    L = s["box"][0]
    f, got = _run(pkg, s["x"], s["y"], s["z"], s["q"], s["tol"], L, s["rcut"])
    p, ref = _oracle("water10k", s["x"], s["y"], s["z"], s["q"], s["tol"], L, s["rcut"], store)
    rep = oracle.error_report(got, ref)
    print("water10k", rep)
    assert rep["force_rms_rel"] <= FORCE_RMS_TOL, rep
    assert rep["energy_rel"] <= ENERGY_TOL, rep
    _ac, cnt, pnt, sidx = oracle.assign(s["x"], s["y"], s["z"], p)
    g_sidx, g_cnt, g_pnt = f.assignment()
    assert np.array_equal(g_sidx, sidx) and np.array_equal(g_cnt, cnt) and np.array_equal(g_pnt, pnt)
    f.close()


def test_direct_coulomb_kernel_matches_oracle(pkg):
    """glst_direct_coulomb (FP64 all pairs on the GPU) against the FP64 host
    oracle; and GLST against it at 30,000 atoms, where the host direct sum is
    slow: the GLST error vs the direct sum is the cubature's (~tol)."""
    x, y, z, q = _water(700, 28.0, 12)
    d = [_dev(a) for a in (x, y, z, q)]
    outs = [torch.empty(len(x), dtype=torch.float64, device="cuda:0") for _ in range(4)]
    pkg.direct_coulomb(*d, *outs)
    torch.cuda.synchronize()
    got = [o.cpu().numpy() for o in outs]
    ref = oracle.coulomb(x, y, z, q)
    rep = oracle.error_report(got, ref)
    assert rep["force_rms_rel"] < 1e-13 and rep["energy_rel"] < 1e-13, rep


@pytest.mark.parametrize("nshards", [2, 3, 5])
def test_node_shards_sum_to_the_full_result(pkg, nshards):
    """Multi-GPU node split on one device: the outputs of shards 0..n-1 add up
    to the unsharded result (the reduction a multi-GPU caller does with NCCL)."""
    n_mol, L, rcut, tol, seed = SYSTEMS["w2000_tol1e-5"]
    x, y, z, q = _water(n_mol, L, seed)
    d = [_dev(a) for a in (x, y, z, q)]
    f, full = _run(pkg, x, y, z, q, tol, L, rcut)
    e_full = f.energy()
    f.close()
    acc = [np.zeros(len(x)) for _ in range(4)]
    e_sum = 0.0
    for s in range(nshards):
        with pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut, shard=(s, nshards)) as g:
            g.calc_ener_force(*d)
            part = g.get_ef()
            e_sum += g.energy()
        for a, b in zip(acc, part):
            a += b
    rep = oracle.error_report(acc, full)
    assert rep["force_rms_rel"] < 1e-12 and rep["energy_rel"] < 1e-12, rep
    assert abs(e_sum - e_full) <= 1e-12 * abs(e_full)


class _DeviceArray:
    """A device pointer of n doubles, readable by torch (CUDA array interface)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2}


def _cell_outputs(f, n):
    """The cell-ordered outputs (the reference's fx()..en()), copied to host."""
    return [torch.as_tensor(_DeviceArray(p, n), device="cuda:0").cpu().numpy().copy() for p in f.cell_outputs()]


@pytest.mark.parametrize("nshards", [2, 4])
def test_reduce_shards_in_library(pkg, nshards):
    """glst_reduce_shards (the reference's reduce of the shards' outputs to
    the first GPU): shards computed on their own streams, summed by shard 0's
    device in shard order -- here all on one device, so the peer reads are
    local; the result in shard 0 equals the unsharded solve, input order, cell
    order and total energy."""
    n_mol, L, rcut, tol, seed = SYSTEMS["w2000_tol1e-5"]
    x, y, z, q = _water(n_mol, L, seed)
    d = [_dev(a) for a in (x, y, z, q)]
    f, full = _run(pkg, x, y, z, q, tol, L, rcut)
    e_full = f.energy()
    cell_full = _cell_outputs(f, len(x))
    f.close()
    streams = [torch.cuda.Stream() for _ in range(nshards)]
    shards = [pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut, shard=(s, nshards)) for s in range(nshards)]
    torch.cuda.synchronize()  # inputs in place before the shards' streams read them
    for sh, st in zip(shards, streams):
        sh.calc_ener_force(*d, stream=st)
    pkg.reduce_shards(shards, streams)
    got = shards[0].get_ef(stream=streams[0])
    rep = oracle.error_report(got, full)
    assert rep["force_rms_rel"] < 1e-12 and rep["energy_rel"] < 1e-12, rep
    assert abs(shards[0].energy(stream=streams[0]) - e_full) <= 1e-12 * abs(e_full)
    torch.cuda.synchronize()
    cell = _cell_outputs(shards[0], len(x))
    assert oracle.error_report(cell, cell_full)["force_rms_rel"] < 1e-12
    for sh in shards:
        sh.close()


def test_autotune_keeps_results(pkg, store):
    """glst_autotune changes launch shapes only: the tuned handle, and a new
    handle of the same shape that inherits the tuning, stay within the parity
    bars of the oracle."""
    n_mol, L, rcut, tol, seed = SYSTEMS["w1000_c1tol"]
    x, y, z, q = _water(n_mol, L, seed)
    d = [_dev(a) for a in (x, y, z, q)]
    p, ref = _oracle("w1000_c1tol", x, y, z, q, tol, L, rcut, store)
    with pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut) as f:
        nb, waves = f.autotune(*d)
        assert nb >= 1 and waves >= 2
        f.calc_ener_force(*d)
        got = f.get_ef()
    rep = oracle.error_report(got, ref)
    assert rep["force_rms_rel"] <= FORCE_RMS_TOL and rep["energy_rel"] <= ENERGY_TOL, rep
    with pkg.GlstForce(len(x), tol, L, L, L, rcut=rcut) as f2:
        f2.calc_ener_force(*d)
        got2 = f2.get_ef()
    rep2 = oracle.error_report(got2, ref)
    assert rep2["force_rms_rel"] <= FORCE_RMS_TOL and rep2["energy_rel"] <= ENERGY_TOL, rep2


def test_init_and_ncell_constructor(pkg, store):
    """glst_force::init re-plans an existing object (src/glst_force.cu:179-327);
    the ncell constructor uses rcut = min(L/n) (src/glst_force.cu:80-95)."""
    n_mol, L, rcut, tol, seed = SYSTEMS["w1000_tol1e-4"]
    x, y, z, q = _water(n_mol, L, seed)
    with pkg.GlstForce(300, 1e-5, 20.0, 20.0, 20.0, rcut=10.0) as f:
        f.init(len(x), tol, L, L, L, rcut)
        f.calc_ener_force(*[_dev(a) for a in (x, y, z, q)])
        got = f.get_ef()
    p, ref = _oracle("w1000_tol1e-4", x, y, z, q, tol, L, rcut, store)
    rep = oracle.error_report(got, ref)
    assert rep["force_rms_rel"] <= FORCE_RMS_TOL and rep["energy_rel"] <= ENERGY_TOL, rep
    with pkg.GlstForce(len(x), tol, L, L, L, ncell=(4, 4, 4)) as g:
        assert tuple(g.info().ncell) == (4, 4, 4)
        assert g.info().cell_dim == L / 4


def test_near_field_three_and_nine_rows(pkg, store):
    """The near field's two launch forms against the oracle at 1e-12, on
    grids with no far field (2 cells along x): 2 x 10 x 15 = 300 cells runs
    three rows of 9 neighbour cells, 2 x 4 x 5 = 40 cells nine rows of 3."""
    rng = np.random.default_rng(17)
    for box, n in (((20.0, 100.0, 150.0), 6000), ((20.0, 40.0, 50.0), 1500)):
        pts = rng.uniform(0.0, 1.0, size=(n, 3)) * np.asarray(box)
        x, y, z = (np.ascontiguousarray(pts[:, i]) for i in range(3))
        q = rng.choice([-0.5, 0.5], n)
        f = pkg.GlstForce(n, 1e-5, *box, rcut=10.0)
        f.calc_ener_force(*[_dev(a) for a in (x, y, z, q)])
        got = f.get_ef()
        assert f.info().has_far_field == 0
        p = planner.make_plan(n, 1e-5, box, 10.0, store)
        rep = oracle.error_report(got, oracle.glst(x, y, z, q, p))
        assert rep["force_rms_rel"] <= 1e-12 and rep["energy_rel"] <= 1e-12, (box, rep)
        f.close()
