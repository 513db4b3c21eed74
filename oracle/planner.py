"""ORACLE (test infrastructure only) -- FP64 restatement of the reference planner.

This module is the checker's copy of the GLST set-up arithmetic.  It is used by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` only; the product computes its own plan in C++
(``csrc/planner.cpp``) and must never import this file.

What it restates (reference file:line):
  * cell grid from box and cutoff in the calculation type CT
    (``src/glst_force.cu:223-241``) and the ncell constructor
    (``src/glst_force.cu:80-95``);
  * alpha groups, shell radii and the Newton inverse of erfc
    (``src/glst_force.cu:1616-1724``);
  * Gauss-Legendre rule selection (``src/cubature.cu:161-402``);
  * spherical t-design selection (``src/cubature.cu:461-523``);
  * node/weight construction (``src/cubature.cu:100-145``).
Everything is FP64, as in the reference's host code.
"""
import math
import os
import struct

import numpy as np

EPS = 2.220446049250313e-16  # std::numeric_limits<double>::epsilon()


def f32(x):
    return float(np.float32(x))


# ----------------------------------------------------------------- cell grid
def cell_grid(box, rcut, ct="double"):
    """(n, cell_dim) following glst_force<CT>::init, src/glst_force.cu:223-241."""
    if ct == "float":
        l = np.float32(rcut)
        n = []
        for L in box:
            Lf = np.float32(L)
            q = np.float32(Lf / l)
            ni = int(q)
            if np.float32(np.float32(ni) * l) < Lf:
                ni += 1
            n.append(ni)
        return tuple(n), float(l)
    l = float(rcut)
    n = []
    for L in box:
        ni = int(float(L) / l)
        if float(ni) * l < float(L):
            ni += 1
        n.append(ni)
    return tuple(n), l


def rcut_from_ncell(box, ncell):
    """rcut = min(L/n), src/glst_force.cu:80-95."""
    r = [float(L) / float(n) for L, n in zip(box, ncell)]
    rc = r[0]
    rc = r[1] if r[1] < rc else rc
    rc = r[2] if r[2] < rc else rc
    return rc


# ----------------------------------------------------------------- alpha groups
def erfc_inv(y, tol):
    """Newton iteration on 1-erf(x)-y from x=0, src/glst_force.cu:1616-1640."""
    rdum = 2.0 / math.sqrt(math.pi)
    x = 0.0
    err = float("inf")
    for _ in range(100000000):
        err = 1.0 - math.erf(x) - y
        if abs(err) < tol:
            break
        deriv = -math.exp(-x * x) * rdum
        x -= err / deriv
    if not abs(err) < tol:
        raise RuntimeError("erfc_inv did not converge")
    return x


def alpha_groups(n, cell_dim, tol):
    """Shell widths, r_max, alpha, z_cut, r_in, r_out (src/glst_force.cu:1643-1724)."""
    widths, rmax, alpha, zcut = [], [], [], []
    width, tot = 1, 0
    remain = max(n) - 2
    lmin = lmax = float(cell_dim)  # cubic cells: cell_dim_x == y == z
    while remain >= 0:
        widths.append(width)
        rmin0 = lmin * float(tot + 1)
        rmax0 = math.sqrt(3.0) * (rmin0 + lmax * float(width + 1))
        rmax.append(rmax0)
        a0 = erfc_inv(tol * rmin0, EPS) / rmin0
        alpha.append(a0)
        zcut.append(erfc_inv(0.5 * math.sqrt(math.pi) / a0 * tol, EPS))
        remain -= width
        tot += width
        if remain < 1:
            break
        w1, w2 = 2 * width, 6 * width
        if remain <= w1:
            width = remain
        elif w1 < remain < w2:
            width = remain // 2
        else:
            width = w1
    r_in, r_out = [], []
    for g, w in enumerate(widths):
        ri = 1 if g == 0 else r_out[g - 1]
        r_in.append(ri)
        r_out.append(ri + w)
    return dict(widths=widths, rmax=rmax, alpha=alpha, zcut=zcut, r_in=r_in, r_out=r_out)


# ----------------------------------------------------------------- Gauss-Legendre
def legendre(x, n):
    """P_n(x), P_n'(x) by the three-term recurrence (src/cubature.cu:161-193)."""
    if n == 0:
        return 1.0, 0.0
    if n == 1:
        return x, 1.0
    p0, p1, p2 = 1.0, x, 0.0
    d1, d2 = 1.0, 0.0
    for i in range(1, n):
        a1 = float(i) + 1.0
        a2 = 2.0 * float(i) + 1.0
        p2 = (a2 * x * p1 - float(i) * p0) / a1
        d2 = a1 * p1 + x * d1
        p0, p1, d1 = p1, p2, d2
    return p2, d2


def legendre_root(x0, n):
    """Newton polish of a root near x0, at most 10 steps (src/cubature.cu:216-238)."""
    dx1, dx2 = 0.0, -1.0
    x = x0
    for _ in range(10):
        p, dp = legendre(x, n)
        dx2 = dx1
        dx1 = p / dp if dp != 0.0 else float("nan")
        if math.isnan(dx1):
            dx1 = 0.0
        x -= dx1
        if abs(dx1) < EPS:
            break
        if abs(dx1 - dx2) < EPS:
            break
    return x


def _walk(x, dx, n, test):
    for _ in range(10):
        p0, d0 = legendre(x, n)
        x += dx
        p1, d1 = legendre(x, n)
        if test(p0, d0, p1, d1):
            return x, True
    return x, False


def gl_roots(n):
    """Non-negative roots of P_n in increasing order (src/cubature.cu:240-351)."""
    if n == 0:
        raise RuntimeError("No roots for n == 0")
    if n == 1:
        return [0.0]
    if n == 2:
        return [1.0 / math.sqrt(3.0)]
    m = n // 2 if n % 2 == 0 else (n + 1) // 2
    dx = 0.1 / float(m + 1)
    x = dx
    roots = []
    passed_extremum = lambda p0, d0, p1, d1: d0 * d1 < 0.0
    if n % 2 == 1:
        roots.append(0.0)
        x, _ = _walk(x, dx, n, passed_extremum)
    # closest approach to zero: step back one dx when |P| starts growing
    for _ in range(10):
        p0, _d = legendre(x, n)
        x += dx
        p1, _d = legendre(x, n)
        if abs(p0) < abs(p1):
            x -= dx
            break
    r0 = legendre_root(x, n)
    roots.append(r0)
    found = 1 if n % 2 == 0 else 2
    x = r0
    dx = 0.2 * r0 if n % 2 == 0 else 0.1 * r0
    while found < m:
        x, _ = _walk(x, dx, n, passed_extremum)
        for _ in range(10):
            p0, _d = legendre(x, n)
            x += dx
            p1, _d = legendre(x, n)
            if abs(p0) < abs(p1):
                x -= dx
                break
        r1 = legendre_root(x, n)
        roots.append(r1)
        x = r1
        dx = 0.1 * (r1 - r0)
        r0 = r1
        found += 1
    return roots


def gl_weights(roots, n):
    """w = 2 / ((1-x^2) P_n'(x)^2) (src/cubature.cu:195-214)."""
    out = []
    for x in roots:
        _p, dp = legendre(x, n)
        out.append(2.0 / ((1.0 - x * x) * dp * dp))
    return out


def select_gauss_legendre(tol, dist, alpha, zcut):
    """Smallest even degree reproducing (pi/2) erf(alpha d) (src/cubature.cu:353-402)."""
    erf0 = 0.5 * math.pi * math.erf(alpha * dist)
    tol0 = 0.5 * math.pi * dist * tol
    for deg in range(2, 325, 2):
        xs = gl_roots(deg)
        ws = gl_weights(xs, deg)
        i0 = 0 if deg % 2 == 0 else 1
        s0 = 0.0 if deg % 2 == 0 else alpha * dist * zcut * ws[0]
        for i in range(i0, len(xs)):
            val = math.exp(-zcut * zcut * xs[i] * xs[i]) * math.sin(2.0 * alpha * dist * zcut * xs[i]) / xs[i]
            s0 += ws[i] * val
        if abs(s0 - erf0) < tol0:
            return deg, xs, ws
    raise RuntimeError("Suitable Gauss-Legendre quadrature could not be found")


# ----------------------------------------------------------------- t-designs
class TDesignStore:
    """Antipodal spherical designs: t -> (m x 3) free half.

    Reads either the project's binary store (``tdesigns.bin``) or a directory in
    the reference's text layout (``ssTTT.NNNNN``, 25-character columns,
    ``src/cubature.cu:422-459``).
    """

    def __init__(self, path):
        self.path = path
        self._cache = {}
        self._files = None
        if os.path.isdir(path):
            self._files = {}
            for name in os.listdir(path):
                full = os.path.join(path, name)
                if len(full) < 9:
                    continue
                try:
                    t = int(full[-9:-6])
                    N = int(full[-5:])
                except ValueError:
                    continue
                self._files.setdefault(t, (full, N // 2))
        else:
            with open(path, "rb") as f:
                data = f.read()
            if data[:8] != b"GLSTTD01":
                raise ValueError("not a t-design store: %s" % path)
            (count,) = struct.unpack_from("<I", data, 8)
            off = 12
            for _ in range(count):
                t, m, _r, _res = struct.unpack_from("<IIId", data, off)
                off += 20
                self._cache[t] = np.frombuffer(data, dtype="<f8", count=3 * m, offset=off).reshape(m, 3).copy()
                off += 24 * m

    def get(self, t):
        if t in self._cache:
            return self._cache[t]
        if self._files is None or t not in self._files:
            raise FileNotFoundError("no spherical t-design of degree %d" % t)
        fname, m = self._files[t]
        pts = np.zeros((m, 3))
        with open(fname) as f:
            for i in range(m):
                line = f.readline()
                pts[i] = [float(line[0:25]), float(line[25:50]), float(line[50:75])]
        self._cache[t] = pts
        return pts


def select_tdesign(store, deg_gl, xs, ws, tol, dist, alpha, zcut):
    """t-design degree search on the three axes (src/cubature.cu:461-523)."""
    zc2 = zcut * zcut
    erf0 = math.erf(alpha * dist) / dist
    n0 = len(xs) // 2
    nmin = -1
    dmin = float("inf")
    i0 = 0 if deg_gl % 2 == 0 else 1
    sm = None
    t_sel = None
    xs_a = np.array(xs)
    ws_a = np.array(ws)
    for j in range(3):
        n = n0
        while n < 162:
            t = 2 * n + 1
            sm = store.get(t)
            t_sel = t
            m = sm.shape[0]
            s0 = 0.0
            comp = sm[:, j]
            for i in range(i0, len(xs)):
                coef = 2.0 * alpha * zcut * dist * xs[i]
                # left-to-right sum in the reference's order (np.cumsum
                # accumulates sequentially, unlike np.sum)
                val = float(np.cumsum(np.cos(coef * comp))[-1])
                x2 = xs[i] * xs[i]
                s0 += ws[i] * math.exp(-zc2 * x2) * val
            s0 *= 4.0 * alpha * zcut / (math.pi * float(m))
            if deg_gl % 2 == 1:
                s0 += 2.0 * alpha * zcut * ws[0] / math.pi
            err = abs(s0 - erf0)
            if err < dmin:
                dmin = err
                nmin = n
            if err < tol:
                n0 = n
                nmin = -2
                break
            n += 1
    if nmin > 0:
        raise RuntimeError("Suitable t-design could not be found")
    return t_sel, sm


# ----------------------------------------------------------------- full plan
class Plan:
    pass


def make_plan(natom, tol, box, rcut, store, ct="double"):
    """Everything glst_force<CT>::init derives from (natom, tol, box, rcut)."""
    p = Plan()
    p.natom = int(natom)
    p.tol = float(tol)
    p.box = tuple(float(b) for b in box)
    p.ct = ct
    p.n, p.cell_dim = cell_grid(box, rcut, ct)
    p.ncell = p.n[0] * p.n[1] * p.n[2]
    g = alpha_groups(p.n, p.cell_dim, tol)
    p.groups = g
    p.ngroup = len(g["widths"])
    p.has_far = all(ni > 2 for ni in p.n)
    kx, ky, kz, w, grp = [], [], [], [], []
    p.gl_degree, p.t_degree, p.n_radial, p.n_dir = [], [], [], []
    for gi in range(p.ngroup):
        a, z, d = g["alpha"][gi], g["zcut"][gi], g["rmax"][gi]
        deg, xs, ws = select_gauss_legendre(tol, d, a, z)
        t, sm = select_tdesign(store, deg, xs, ws, tol, d, a, z)
        p.gl_degree.append(deg)
        p.t_degree.append(t)
        p.n_radial.append(len(xs))
        p.n_dir.append(sm.shape[0])
        msz = float(sm.shape[0])
        zc2 = z * z
        for i in range(len(xs)):
            sc = 2.0 * a * z * xs[i]
            wi = 4.0 * a * z * ws[i] * math.exp(-zc2 * xs[i] * xs[i]) / (math.pi * msz)
            # same association order as src/cubature.cu:129-137
            kx.extend([2.0 * a * z * xs[i] * s for s in sm[:, 0]])
            ky.extend([2.0 * a * z * xs[i] * s for s in sm[:, 1]])
            kz.extend([2.0 * a * z * xs[i] * s for s in sm[:, 2]])
            w.extend([wi] * sm.shape[0])
            grp.extend([gi] * sm.shape[0])
    p.kx = np.array(kx)
    p.ky = np.array(ky)
    p.kz = np.array(kz)
    p.w = np.array(w)
    p.group = np.array(grp, dtype=np.uint32)
    p.K = p.kx.size
    if ct == "float":
        p.kx, p.ky, p.kz, p.w = (a.astype(np.float32).astype(np.float64) for a in (p.kx, p.ky, p.kz, p.w))
    return p
