"""glst_b200 -- Python mirror of the reference's ``glst_force<CT>`` object.

The compute path is the CUDA engine in ``libglst_b200.so`` (csrc/, built for
sm_100a); this module only binds its C-ABI (``include/glst_c.h``) with ctypes
and mirrors the reference's C++ interface (include/glst_force.hcu:24-125):

    f = GlstForce(natom, tol, box_x, box_y, box_z, rcut=10.0, ct="double")
    f.calc_ener_force(d_rx, d_ry, d_rz, d_qc)      # device FP64 arrays
    fx, fy, fz, en = f.get_ef()                     # input order, host
    e_total = f.energy()                            # 0.5 * sum(en)

Device arrays are anything with ``data_ptr()`` (a torch CUDA tensor) or raw
integer device addresses.  Errors raise ``GlstError`` (the reference throws
std::runtime_error).  There is no CPU fallback: if the library cannot be
loaded, importing this package fails.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libglst_b200.so")
TDESIGN_STORE = os.path.join(_HERE, "data", "tdesigns.bin")

__all__ = ["GlstForce", "GlstBatch", "GlstServer", "GlstError", "load_library", "plan", "LIB_PATH", "TDESIGN_STORE", "set_tdesign_path"]


class GlstError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (status %d)" % (message, status))
        self.status = status


class GlstInfo(ctypes.Structure):
    _fields_ = [
        ("natom", ctypes.c_uint32),
        ("ncell", ctypes.c_uint32 * 3),
        ("ncell_total", ctypes.c_uint32),
        ("cell_dim", ctypes.c_double),
        ("ngroup", ctypes.c_uint32),
        ("num_nodes", ctypes.c_uint32),
        ("has_far_field", ctypes.c_uint32),
        ("group_nodes", ctypes.c_uint32 * 16),
        ("group_gl_degree", ctypes.c_uint32 * 16),
        ("group_t_degree", ctypes.c_uint32 * 16),
        ("group_alpha", ctypes.c_double * 16),
        ("group_zcut", ctypes.c_double * 16),
        ("group_rmax", ctypes.c_double * 16),
        ("group_r_in", ctypes.c_uint32 * 16),
        ("group_r_out", ctypes.c_uint32 * 16),
        ("device_bytes", ctypes.c_uint64),
        ("kernels_per_compute", ctypes.c_uint32),
        ("node_stages", ctypes.c_uint32),
        ("shell_sums_form", ctypes.c_uint32),
        ("gather_variant", ctypes.c_uint32),
        ("sf_max_npt", ctypes.c_uint32),
    ]


# Every entry point of include/glst_c.h with its ctypes signature.
_P, _D, _U32, _I = ctypes.c_void_p, ctypes.c_double, ctypes.c_uint32, ctypes.c_int
_DP = ctypes.POINTER(ctypes.c_double)
_SIGNATURES = {
    "glst_set_tdesign_path": (_I, [ctypes.c_char_p]),
    "glst_create": (_I, [ctypes.POINTER(_P), _U32, _D, _D, _D, _D, _D, _I]),
    "glst_create_shard": (_I, [ctypes.POINTER(_P), _U32, _D, _D, _D, _D, _D, _I, _U32, _U32]),
    "glst_create_ncell": (_I, [ctypes.POINTER(_P), _U32, _D, _D, _D, _D, _U32, _U32, _U32, _I]),
    "glst_init": (_I, [_P, _U32, _D, _D, _D, _D, _D]),
    "glst_destroy": (_I, [_P]),
    "glst_compute": (_I, [_P, _P, _P, _P, _P, _P]),
    "glst_assign_atoms": (_I, [_P, _P, _P, _P, _P, _P]),
    "glst_calc_sf": (_I, [_P, _P]),
    "glst_sum_rmt_sf": (_I, [_P, _P]),
    "glst_calc_lr_ef": (_I, [_P, _P]),
    "glst_calc_sr_ef": (_I, [_P, _P]),
    "glst_comm_ef": (_I, [_P, _P]),
    "glst_get_ef": (_I, [_P, _P, _P, _P, _P, _I, _P]),
    "glst_cell_outputs": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "glst_energy": (_I, [_P, _DP, _P]),
    "glst_compute_host": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "glst_get_assignment": (_I, [_P, _P, _P, _P]),
    "glst_get_info": (_I, [_P, ctypes.POINTER(GlstInfo)]),
    "glst_get_nodes": (_I, [_P, _P, _P, _P, _P, _P]),
    "glst_check": (_I, [_P, _P]),
    "glst_get_far_field": (_I, [_P, _P, _P, _P, _P, _P]),
    "glst_reduce_shards": (_I, [_P, _U32, _P]),
    "glst_plan": (_I, [_U32, _D, _D, _D, _D, _D, _I, ctypes.POINTER(GlstInfo), _P, _P, _P, _P, _P]),
    "glst_max_atoms_per_cell": (_U32, []),
    "glst_measure_pipe_peaks": (_I, [_DP, _DP]),
    "glst_autotune": (_I, [_P, _P, _P, _P, _P, _P, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "glst_direct_coulomb": (_I, [_U32, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "glst_batch_create": (_I, [ctypes.POINTER(_P), _U32, _P, _P, _P, _P, _I, _U32]),
    "glst_batch_destroy": (_I, [_P]),
    "glst_batch_compute": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "glst_batch_energies": (_I, [_P, _P, _P]),
    "glst_batch_system": (_I, [_P, _U32, ctypes.POINTER(_P)]),
    "glst_server_create": (_I, [ctypes.POINTER(_P), ctypes.c_uint64, _U32]),
    "glst_server_destroy": (_I, [_P]),
    "glst_server_submit": (_I, [_P, ctypes.c_uint64, _U32, _D, _D, _D, _D, _D, _P, _P, _P, _P,
                                ctypes.POINTER(ctypes.c_uint64)]),
    "glst_server_wait": (_I, [_P, ctypes.c_uint64, _P, _P, _P, _P, _DP, _DP, _D]),
    "glst_server_get_stats": (_I, [_P, _P]),
    "glst_near_field_noalloc": (_I, [_U32, _P, _P, _P, _P, _D, _D, _D, _D, _I, _P, _P, _P, _P, _P]),
    "glst_last_error": (ctypes.c_char_p, []),
    "glst_status_string": (ctypes.c_char_p, [_I]),
    "glst_version": (ctypes.c_char_p, []),
}

_lib = None


def load_library(path=None):
    """Load (once) the CUDA engine.  Raises OSError if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError("libglst_b200.so not found at %s: run build.py (nvcc, sm_100a) first" % p)
    lib = ctypes.CDLL(p)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _check(status):
    if status != 0:
        lib = load_library()
        raise GlstError(status, lib.glst_last_error().decode(errors="replace"))


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    raise TypeError("expected a device tensor, numpy array or integer address")


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return s
    if hasattr(s, "cuda_stream"):
        return s.cuda_stream
    raise TypeError("expected a torch.cuda.Stream or an integer cudaStream_t")


def set_tdesign_path(path):
    """Process-wide t-design source: binary store or reference-layout directory."""
    _check(load_library().glst_set_tdesign_path(None if path is None else path.encode()))


def plan(natom, tol, box, rcut, ct="double", with_nodes=True):
    """Host-only plan (no GPU needed): (GlstInfo, (kx, ky, kz, w, group) or None)."""
    lib = load_library()
    inf = GlstInfo()
    cti = 1 if ct == "float" else 0
    args = (int(natom), float(tol), float(box[0]), float(box[1]), float(box[2]), float(rcut), cti,
            ctypes.byref(inf))
    _check(lib.glst_plan(*args, None, None, None, None, None))
    if not with_nodes:
        return inf, None
    K = inf.num_nodes
    arrs = [np.empty(K) for _ in range(4)] + [np.empty(K, dtype=np.uint32)]
    _check(lib.glst_plan(*args, *[a.ctypes.data for a in arrs]))
    return inf, tuple(arrs)


def direct_coulomb(x, y, z, q, fx, fy, fz, en, stream=None):
    """FP64 all-pairs Coulomb on the GPU (device arrays, input order)."""
    n = x.numel() if hasattr(x, "numel") else len(x)
    _check(load_library().glst_direct_coulomb(int(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(fx), _ptr(fy),
                                              _ptr(fz), _ptr(en), _stream(stream)))


def measure_pipe_peaks():
    """(MUFU sin+cos results/s, FP32 FMA/s) of the current device."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(load_library().glst_measure_pipe_peaks(ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


class GlstForce:
    """One GLST system on the current CUDA device (mirrors glst_force<CT>)."""

    def __init__(self, natom, tol, box_dim_x, box_dim_y, box_dim_z, rcut=None, ncell=None, ct="double",
                 shard=None):
        self._lib = load_library()
        self._h = ctypes.c_void_p()
        if ct not in ("double", "float"):
            raise ValueError("ct must be 'double' or 'float'")
        cti = 1 if ct == "float" else 0
        self.ct = ct
        if (rcut is None) == (ncell is None):
            raise ValueError("give exactly one of rcut or ncell")
        if shard is not None:
            if rcut is None:
                raise ValueError("a shard needs rcut")
            s, n = shard
            _check(self._lib.glst_create_shard(ctypes.byref(self._h), int(natom), float(tol), float(box_dim_x),
                                               float(box_dim_y), float(box_dim_z), float(rcut), cti, int(s), int(n)))
        elif rcut is not None:
            _check(self._lib.glst_create(ctypes.byref(self._h), int(natom), float(tol), float(box_dim_x),
                                         float(box_dim_y), float(box_dim_z), float(rcut), cti))
        else:
            nx, ny, nz = ncell
            _check(self._lib.glst_create_ncell(ctypes.byref(self._h), int(natom), float(tol), float(box_dim_x),
                                               float(box_dim_y), float(box_dim_z), int(nx), int(ny), int(nz), cti))
        self.natom = int(natom)
        self._info = None

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if self._h:
            self._lib.glst_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init(self, natom, tol, box_dim_x, box_dim_y, box_dim_z, rcut):
        _check(self._lib.glst_init(self._h, int(natom), float(tol), float(box_dim_x), float(box_dim_y),
                                   float(box_dim_z), float(rcut)))
        self.natom = int(natom)
        self._info = None

    # -- compute (src/glst_force.cu:1604-1614 and the six phases) -----------
    def calc_ener_force(self, d_rx, d_ry, d_rz, d_qc, stream=None):
        _check(self._lib.glst_compute(self._h, _ptr(d_rx), _ptr(d_ry), _ptr(d_rz), _ptr(d_qc), _stream(stream)))

    def autotune(self, d_rx, d_ry, d_rz, d_qc, stream=None):
        """Pick the shell-sum and long-range launch shapes by timing them on
        these inputs; returns (nodes per shell CTA, long-range waves)."""
        a, b = ctypes.c_uint32(), ctypes.c_uint32()
        _check(self._lib.glst_autotune(self._h, _ptr(d_rx), _ptr(d_ry), _ptr(d_rz), _ptr(d_qc), _stream(stream),
                                       ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def assign_atoms(self, d_rx, d_ry, d_rz, d_qc, stream=None):
        _check(self._lib.glst_assign_atoms(self._h, _ptr(d_rx), _ptr(d_ry), _ptr(d_rz), _ptr(d_qc),
                                           _stream(stream)))

    def calc_sf(self, stream=None):
        _check(self._lib.glst_calc_sf(self._h, _stream(stream)))

    def sum_rmt_sf(self, stream=None):
        _check(self._lib.glst_sum_rmt_sf(self._h, _stream(stream)))

    def calc_lr_ef(self, stream=None):
        _check(self._lib.glst_calc_lr_ef(self._h, _stream(stream)))

    def calc_sr_ef(self, stream=None):
        _check(self._lib.glst_calc_sr_ef(self._h, _stream(stream)))

    def comm_ef(self, stream=None):
        _check(self._lib.glst_comm_ef(self._h, _stream(stream)))

    def compute_host(self, x, y, z, q, stream=None):
        """End to end from host arrays; returns (fx, fy, fz, en) in input order."""
        n = self.natom
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
        outs = [np.empty(n) for _ in range(4)]
        _check(self._lib.glst_compute_host(self._h, *[a.ctypes.data for a in arrs],
                                           *[o.ctypes.data for o in outs], _stream(stream)))
        return tuple(outs)

    # -- results -----------------------------------------------------------
    def get_ef(self, fx=None, fy=None, fz=None, en=None, stream=None):
        """Input-order forces and energies.  With no arguments: host numpy
        arrays.  With device tensors: filled in place, stream ordered."""
        if fx is None and fy is None and fz is None and en is None:
            outs = [np.empty(self.natom) for _ in range(4)]
            _check(self._lib.glst_get_ef(self._h, *[o.ctypes.data for o in outs], 0, _stream(stream)))
            return tuple(outs)
        _check(self._lib.glst_get_ef(self._h, _ptr(fx), _ptr(fy), _ptr(fz), _ptr(en), 1, _stream(stream)))
        return fx, fy, fz, en

    def cell_outputs(self):
        """Device addresses of the cell-ordered fx, fy, fz, en (reference fx()...en())."""
        ps = [ctypes.c_void_p() for _ in range(4)]
        _check(self._lib.glst_cell_outputs(self._h, *[ctypes.byref(p) for p in ps]))
        return tuple(p.value for p in ps)

    def energy(self, stream=None):
        e = ctypes.c_double()
        _check(self._lib.glst_energy(self._h, ctypes.byref(e), _stream(stream)))
        return e.value

    def check(self, stream=None):
        _check(self._lib.glst_check(self._h, _stream(stream)))

    def assignment(self):
        info = self.info()
        sidx = np.empty(self.natom, dtype=np.uint32)
        cnt = np.empty(info.ncell_total, dtype=np.uint32)
        pnt = np.empty(info.ncell_total, dtype=np.uint32)
        _check(self._lib.glst_get_assignment(self._h, sidx.ctypes.data, cnt.ctypes.data, pnt.ctypes.data))
        return sidx, cnt, pnt

    def info(self):
        if self._info is None:
            inf = GlstInfo()
            _check(self._lib.glst_get_info(self._h, ctypes.byref(inf)))
            self._info = inf
        return self._info

    def far_field(self, stream=None):
        """(sf, rmt): complex128 arrays [ncell, K] of the last assigned
        positions, in the reference's layout and definitions (its sf_re_/sf_im_
        after calc_sf and rmt_sum_re_/rmt_sum_im_ after sum_rmt_sf), nodes in
        the order of ``nodes()``."""
        inf = self.info()
        C, K = inf.ncell_total, inf.num_nodes
        arrs = [np.empty((C, K)) for _ in range(4)]
        _check(self._lib.glst_get_far_field(self._h, *[a.ctypes.data for a in arrs], _stream(stream)))
        return arrs[0] + 1j * arrs[1], arrs[2] + 1j * arrs[3]

    def nodes(self):
        K = self.info().num_nodes
        arrs = [np.empty(K) for _ in range(4)] + [np.empty(K, dtype=np.uint32)]
        _check(self._lib.glst_get_nodes(self._h, *[a.ctypes.data for a in arrs]))
        return tuple(arrs)


def reduce_shards(shards, streams=None):
    """Sum the outputs of shard handles 0..n-1 of one system into shard 0's
    (glst_reduce_shards: the reference's reduce to the first GPU).  shards:
    GlstForce objects made with shard=(s, n), each computed on streams[s]
    (default: the legacy stream)."""
    lib = load_library()
    n = len(shards)
    hs = (ctypes.c_void_p * n)(*[s._h.value for s in shards])
    sts = (ctypes.c_void_p * n)(*[_stream(s) for s in (streams or [None] * n)])
    _check(lib.glst_reduce_shards(hs, n, sts))


class GlstBatch:
    """Many independent systems solved together (glst_batch_* of the C-ABI).

    systems: sequence of dicts with natom, tol, box (3), rcut.  Inputs and
    outputs are concatenated in system order (``offsets`` gives the starts).
    ``compute(..., plain=False)`` runs one captured CUDA graph over all
    systems (their launch sequences on parallel branches; ``mode="worklist"``:
    one launch per phase over a work list of every system's blocks);
    ``plain=True`` solves them one after another (baseline).
    """

    def __init__(self, systems, ct="double", nstreams=16):
        self._lib = load_library()
        self._b = ctypes.c_void_p()
        n = len(systems)
        natom = np.array([s["natom"] for s in systems], dtype=np.uint32)
        tol = np.array([s["tol"] for s in systems], dtype=np.float64)
        box = np.array([list(s["box"]) for s in systems], dtype=np.float64).reshape(-1)
        rcut = np.array([s["rcut"] for s in systems], dtype=np.float64)
        _check(self._lib.glst_batch_create(ctypes.byref(self._b), n, natom.ctypes.data, tol.ctypes.data,
                                           box.ctypes.data, rcut.ctypes.data, 1 if ct == "float" else 0,
                                           int(nstreams)))
        self.nsys = n
        self.natom = natom
        self.offsets = np.concatenate([[0], np.cumsum(natom.astype(np.int64))])

    def close(self):
        if self._b:
            self._lib.glst_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    MODES = {"branches": 0, "plain": 1, "worklist": 2}

    def compute(self, x, y, z, q, fx, fy, fz, en, plain=False, stream=None, mode=None):
        """mode: "branches" (default; every system its own launch sequence
        on parallel branches of one captured graph), "plain" (one system
        after another; also plain=True), "worklist" (one launch per phase for
        every system that fits the work-list kernels, the others on
        branches)."""
        m = self.MODES[mode] if mode is not None else (1 if plain else 0)
        _check(self._lib.glst_batch_compute(self._b, _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(fx), _ptr(fy),
                                            _ptr(fz), _ptr(en), m, _stream(stream)))

    def energies(self, stream=None):
        e = np.empty(self.nsys)
        _check(self._lib.glst_batch_energies(self._b, e.ctypes.data, _stream(stream)))
        return e


class GlstServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("evictions", ctypes.c_uint64),
                ("systems_created", ctypes.c_uint64), ("resident_bytes", ctypes.c_uint64),
                ("peak_resident_bytes", ctypes.c_uint64), ("resident_systems", ctypes.c_uint32),
                ("in_flight", ctypes.c_uint32)]


class GlstServer:
    """Continuous-batching request server over the engine (glst_server_*).

    ``submit`` queues an energy+force request (host arrays are copied) and
    returns a ticket; ``wait`` returns (fx, fy, fz, en, energy, latency_us).
    ``key`` names a resident system whose plan and buffers are reused when
    the same key comes back with the same natom, tol, box and rcut."""

    def __init__(self, budget_bytes, nslots=8):
        self._lib = load_library()
        self._s = ctypes.c_void_p()
        _check(self._lib.glst_server_create(ctypes.byref(self._s), int(budget_bytes), int(nslots)))

    def close(self):
        if self._s:
            self._lib.glst_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, key, x, y, z, q, tol, box, rcut):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
        t = ctypes.c_uint64()
        _check(self._lib.glst_server_submit(self._s, int(key), len(arrs[0]), float(tol), float(box[0]),
                                            float(box[1]), float(box[2]), float(rcut),
                                            *[a.ctypes.data for a in arrs], ctypes.byref(t)))
        return t.value, len(arrs[0])

    def wait(self, ticket, timeout_ms=-1.0):
        t, n = ticket
        outs = [np.empty(n) for _ in range(4)]
        e, lat = ctypes.c_double(), ctypes.c_double()
        _check(self._lib.glst_server_wait(self._s, t, *[o.ctypes.data for o in outs], ctypes.byref(e),
                                          ctypes.byref(lat), float(timeout_ms)))
        return (*outs, e.value, lat.value)

    def stats(self):
        st = GlstServerStats()
        _check(self._lib.glst_server_get_stats(self._s, ctypes.byref(st)))
        return st
