"""ORACLE (test infrastructure only): ctypes front end of glst_oracle.c.

``make_plan`` comes from planner.py (the FP64 restatement of the reference's
set-up); ``glst`` runs the FP64 GLST sum of the reference's double path on the
host (OpenMP); ``coulomb`` is the all-pairs FP64 direct sum.
"""
import ctypes
import os
import subprocess

import numpy as np

from .planner import TDesignStore, make_plan, rcut_from_ncell  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libglst_oracle.so")


class _Plan(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_uint32), ("ny", ctypes.c_uint32), ("nz", ctypes.c_uint32),
        ("cell_dim", ctypes.c_double), ("ct_float", ctypes.c_int), ("K", ctypes.c_uint32),
        ("kx", ctypes.c_void_p), ("ky", ctypes.c_void_p), ("kz", ctypes.c_void_p), ("w", ctypes.c_void_p),
        ("group", ctypes.c_void_p), ("ngroup", ctypes.c_uint32),
        ("r_in", ctypes.c_void_p), ("r_out", ctypes.c_void_p), ("has_far", ctypes.c_int),
    ]


_lib = None


def build():
    src = os.path.join(HERE, "glst_oracle.c")
    if not os.path.exists(SO) or os.path.getmtime(SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "libglst_oracle.so"], check=True)
    return SO


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(SO)
        _lib.oracle_glst.restype = ctypes.c_int
        _lib.oracle_far_arrays.restype = ctypes.c_int
        _lib.oracle_assign.restype = ctypes.c_int
        _lib.oracle_num_threads.restype = ctypes.c_int
    return _lib


def num_threads():
    return lib().oracle_num_threads()


class _Keep:
    """Holds the numpy arrays a ctypes plan points into."""


def _cplan(plan):
    keep = _Keep()
    keep.kx = np.ascontiguousarray(plan.kx, dtype=np.float64)
    keep.ky = np.ascontiguousarray(plan.ky, dtype=np.float64)
    keep.kz = np.ascontiguousarray(plan.kz, dtype=np.float64)
    keep.w = np.ascontiguousarray(plan.w, dtype=np.float64)
    keep.g = np.ascontiguousarray(plan.group, dtype=np.uint32)
    keep.ri = np.ascontiguousarray(plan.groups["r_in"] or [1], dtype=np.uint32)
    keep.ro = np.ascontiguousarray(plan.groups["r_out"] or [2], dtype=np.uint32)
    cp = _Plan(plan.n[0], plan.n[1], plan.n[2], plan.cell_dim, 1 if plan.ct == "float" else 0, plan.K,
               keep.kx.ctypes.data, keep.ky.ctypes.data, keep.kz.ctypes.data, keep.w.ctypes.data,
               keep.g.ctypes.data, plan.ngroup, keep.ri.ctypes.data, keep.ro.ctypes.data,
               1 if plan.has_far else 0)
    return cp, keep


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def assign(x, y, z, plan):
    """(atom_cell, cell_count, cell_point, sorted_idx), reference semantics."""
    n = len(x)
    cp, keep = _cplan(plan)
    x, y, z = _d(x), _d(y), _d(z)
    ac = np.empty(n, dtype=np.uint32)
    cnt = np.empty(plan.ncell, dtype=np.uint32)
    pnt = np.empty(plan.ncell, dtype=np.uint32)
    sidx = np.empty(n, dtype=np.uint32)
    lib().oracle_assign(ctypes.c_uint32(n), x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p),
                        z.ctypes.data_as(ctypes.c_void_p), ctypes.byref(cp), ac.ctypes.data_as(ctypes.c_void_p),
                        cnt.ctypes.data_as(ctypes.c_void_p), pnt.ctypes.data_as(ctypes.c_void_p),
                        sidx.ctypes.data_as(ctypes.c_void_p))
    return ac, cnt, pnt, sidx


def glst(x, y, z, q, plan, k0=0, k1=None, far=True, sr=True):
    """FP64 GLST energies/forces in input order (reference double path)."""
    n = len(x)
    cp, keep = _cplan(plan)
    x, y, z, q = _d(x), _d(y), _d(z), _d(q)
    out = [np.empty(n) for _ in range(4)]
    k1 = plan.K if k1 is None else k1
    V = ctypes.c_void_p
    rc = lib().oracle_glst(ctypes.c_uint32(n), x.ctypes.data_as(V), y.ctypes.data_as(V), z.ctypes.data_as(V),
                           q.ctypes.data_as(V), ctypes.byref(cp), ctypes.c_uint32(k0), ctypes.c_uint32(k1),
                           ctypes.c_int(1 if far else 0), ctypes.c_int(1 if sr else 0),
                           *[o.ctypes.data_as(V) for o in out])
    if rc != 0:
        raise MemoryError("oracle_glst failed")
    return tuple(out)


def far_arrays(x, y, z, q, plan):
    """The reference's per-phase far-field arrays (FP64), complex [ncell, K]:
    sf = sum_j q_j e^{-ik.r_j} after calc_sf (src/glst_force.cu:601-664) and
    rmt = w times the shell sum after sum_rmt_sf (:702-913)."""
    n = len(x)
    cp, keep = _cplan(plan)
    x, y, z, q = _d(x), _d(y), _d(z), _d(q)
    C, K = plan.ncell, plan.K
    out = [np.empty((C, K)) for _ in range(4)]
    V = ctypes.c_void_p
    rc = lib().oracle_far_arrays(ctypes.c_uint32(n), x.ctypes.data_as(V), y.ctypes.data_as(V), z.ctypes.data_as(V),
                                 q.ctypes.data_as(V), ctypes.byref(cp), *[o.ctypes.data_as(V) for o in out])
    if rc != 0:
        raise MemoryError("oracle_far_arrays failed")
    return out[0] + 1j * out[1], out[2] + 1j * out[3]


def coulomb(x, y, z, q):
    n = len(x)
    x, y, z, q = _d(x), _d(y), _d(z), _d(q)
    out = [np.empty(n) for _ in range(4)]
    V = ctypes.c_void_p
    lib().oracle_coulomb(ctypes.c_uint32(n), x.ctypes.data_as(V), y.ctypes.data_as(V), z.ctypes.data_as(V),
                         q.ctypes.data_as(V), *[o.ctypes.data_as(V) for o in out])
    return tuple(out)


def error_report(f_test, f_ref):
    """Relative force RMS, max relative force error and energy relative error.

    force RMS: sqrt(sum |dF|^2 / sum |F_ref|^2);  energy: |dE| / |E_ref| with
    E = 0.5 * sum(en).  f_* = (fx, fy, fz, en) arrays.
    """
    dF2 = sum(np.sum((np.asarray(a) - np.asarray(b)) ** 2) for a, b in zip(f_test[:3], f_ref[:3]))
    F2 = sum(np.sum(np.asarray(b) ** 2) for b in f_ref[:3])
    fmag = np.sqrt(sum(np.asarray(b) ** 2 for b in f_ref[:3]))
    dmag = np.sqrt(sum((np.asarray(a) - np.asarray(b)) ** 2 for a, b in zip(f_test[:3], f_ref[:3])))
    e_t = 0.5 * float(np.sum(f_test[3]))
    e_r = 0.5 * float(np.sum(f_ref[3]))
    return dict(force_rms_rel=float(np.sqrt(dF2 / F2)) if F2 > 0 else 0.0,
                force_max_rel=float(np.max(dmag) / np.sqrt(F2 / len(fmag))) if F2 > 0 else 0.0,
                energy_rel=abs(e_t - e_r) / abs(e_r) if e_r != 0 else abs(e_t - e_r),
                energy=e_t, energy_ref=e_r)
