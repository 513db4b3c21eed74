"""Allocation-free near field, called through the C-ABI (GPU).

Some callers cannot allocate device memory at the moment they need forces:
code running while a CUDA stream is being captured into a graph (cudaMalloc
is not permitted during capture), and MD engines or plugins whose host owns
the whole device through its own memory pool.  For them the library has
glst_near_field_noalloc, whose working memory is one fixed-size file-scope
device array; the caller passes only inputs and outputs.

Its result must equal the regular entry point's wherever both compute the
same thing: on a grid with at most two cells along some axis the reference --
and so glst_compute -- has no far field and returns exactly the near field.
Calls in a row on systems of different sizes -- a larger one after a smaller
one, then a smaller one after the larger (so leftovers of a larger call in
the shared array would show) -- and a call binning in float arithmetic
(glst_force<float>'s cell assignment) are each compared with glst_compute at
the tolerances of the other parity tests.  This file is named to be collected
last.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FORCE_RMS_TOL = 1e-5
ENERGY_TOL = 1e-7
GLST_ERR_SIZE = 7


def _dev(a):
    return torch.tensor(np.asarray(a), dtype=torch.float64, device="cuda:0")


def _noalloc(lib, x, y, z, q, box, rcut, ct=0):
    n = len(x)
    ins = [_dev(a) for a in (x, y, z, q)]
    outs = [torch.full((n,), float("nan"), dtype=torch.float64, device="cuda:0") for _ in range(4)]
    st = lib.glst_near_field_noalloc(ctypes.c_uint32(n), *[ctypes.c_void_p(t.data_ptr()) for t in ins],
                                     ctypes.c_double(box[0]), ctypes.c_double(box[1]), ctypes.c_double(box[2]),
                                     ctypes.c_double(rcut), ctypes.c_int(ct),
                                     *[ctypes.c_void_p(t.data_ptr()) for t in outs], None)
    assert st == 0, lib.glst_last_error()
    torch.cuda.synchronize()
    return tuple(t.cpu().numpy() for t in outs)


def _regular(pkg, x, y, z, q, box, rcut, ct=0):
    with pkg.GlstForce(len(x), 1e-6, *box, rcut=rcut, ct="float" if ct else "double") as f:
        assert f.info().has_far_field == 0
        f.calc_ener_force(*[_dev(a) for a in (x, y, z, q)])
        return f.get_ef()


def _systems():
    from glst_b200 import systems
    a = systems.water_box(300, 19.5, seed=21)                      # 2 x 2 x 2 cells
    rng = np.random.default_rng(22)
    n = 4000
    pts = rng.uniform(0.0, 1.0, size=(n, 3)) * np.array([40.0, 40.0, 15.0])   # 4 x 4 x 2 cells
    q = rng.choice([-0.5, 0.5], n)
    b = tuple(np.ascontiguousarray(pts[:, i]) for i in range(3)) + (q,)
    c = systems.water_box(40, 9.5, seed=23)                       # 1 x 1 x 1 cell
    # small, larger (more atoms and cells), then smaller again; the last
    # bins in float arithmetic (glst_force<float>)
    return [(a, (19.5, 19.5, 19.5), 0), (b, (40.0, 40.0, 15.0), 0), (c, (9.5, 9.5, 9.5), 0),
            (a, (19.5, 19.5, 19.5), 1)]


def test_noalloc_matches_regular_entry_point_in_a_row(pkg):
    lib = pkg.load_library()
    for (x, y, z, q), box, ct in _systems():
        got = _noalloc(lib, x, y, z, q, box, 10.0, ct=ct)
        ref = _regular(pkg, x, y, z, q, box, 10.0, ct=ct)
        assert all(np.isfinite(a).all() for a in got)
        rep = oracle.error_report(got, ref)
        assert rep["force_rms_rel"] <= FORCE_RMS_TOL, rep
        assert rep["energy_rel"] <= ENERGY_TOL, rep


def test_noalloc_rejects_boxes_beyond_its_cell_limit(pkg):
    """A box / rcut ratio beyond the cell limit along one axis (or not
    finite) is rejected before any integer conversion."""
    lib = pkg.load_library()
    d = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(d.data_ptr())
    for bx in (1e12, float("inf")):
        st = lib.glst_near_field_noalloc(ctypes.c_uint32(4), p, p, p, p, ctypes.c_double(bx),
                                         ctypes.c_double(10.0), ctypes.c_double(10.0), ctypes.c_double(5.0),
                                         ctypes.c_int(0), p, p, p, p, None)
        assert st == GLST_ERR_SIZE


def test_noalloc_rejects_sizes_beyond_its_limit(pkg):
    lib = pkg.load_library()
    n = 32768 + 1  # GLST_NOALLOC_MAX_ATOMS + 1
    d = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(d.data_ptr())
    st = lib.glst_near_field_noalloc(ctypes.c_uint32(n), p, p, p, p, ctypes.c_double(10.0),
                                     ctypes.c_double(10.0), ctypes.c_double(10.0), ctypes.c_double(5.0),
                                     ctypes.c_int(0), p, p, p, p, None)
    assert st == GLST_ERR_SIZE
    assert b"allocation-free limit" in lib.glst_last_error()
