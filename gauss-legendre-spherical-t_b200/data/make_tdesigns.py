"""Generate equal-weight antipodal spherical t-designs for the GLST cubature.

Why this exists
---------------
The reference reads Womersley-style symmetric spherical designs from a
directory ``SS31-Mar-2016/`` (``src/cubature.cu:423-459``, ``:490``) that it
does not ship.  This script computes our own designs, numerically, by the
published variational characterisation of Sloan & Womersley ("A variational
characterisation of spherical designs", J. Approx. Theory 159 (2009)):
a point set X on S^2 is a t-design iff every spherical harmonic of degree
1 <= l <= t sums to zero over X.  For an antipodal set X = {+-p_i} every odd
degree vanishes by symmetry, so with t odd the conditions are

    r_{l,mu}(p) = sqrt(4 pi)/m * sum_i Y_{l,mu}(p_i) = 0,   l = 2,4,...,t-1.

That is E = 2s^2 + 3s equations (t = 2s+1) in 2m unknowns (two tangent
coordinates per free point).  We take m0 = ceil((E+3)/2) (the +3 accounts for
the rotational invariance) plus a 5% margin of free points, which keeps the
Jacobian well conditioned (near-square systems converge several times more
slowly from a spiral start), and solve r(p) = 0 with
Levenberg-Marquardt in minimum-norm form, dp = -J^T (J J^T + lam I)^-1 r,
started from a spherical Fibonacci lattice on the upper hemisphere.

Output
------
``tdesigns.bin`` (little endian):  b"GLSTTD01", u32 count, then per design
u32 t, u32 m, u32 reserved, f64 residual, then m x 3 f64 unit vectors (the free
half; the full design is {p_i} U {-p_i}, N = 2m points).  The library reads this
store directly; ``write_reference_dir`` renders it in the reference's text
layout (file ``ssTTT.NNNNN``, three 25-character columns per line, the free half
first and the antipodes after it) so the reference can consume identical nodes.

Usage:  python make_tdesigns.py [--tmax 141] [--out tdesigns.bin]
The run is resumable: degrees already present in the output are kept.
"""
import argparse
import math
import os
import struct
import sys
import time

import numpy as np
from scipy.linalg import cho_factor, cho_solve
from scipy.linalg.blas import dsyrk

MAGIC = b"GLSTTD01"
MARGIN_FRACTION = 0.05


def n_equations(t):
    s = (t - 1) // 2
    return 2 * s * s + 3 * s


def n_free_points(t):
    if t == 1:
        return 1
    m0 = (n_equations(t) + 3 + 1) // 2
    return m0 + 2 + int(math.ceil(MARGIN_FRACTION * m0))


def fibonacci_hemisphere(m):
    """m points on the upper hemisphere, equal-area spiral (no antipodal pairs)."""
    i = np.arange(m, dtype=np.float64)
    z = 1.0 - (i + 0.5) / m
    golden = math.pi * (3.0 - math.sqrt(5.0))
    phi = np.mod(i * golden, 2.0 * math.pi)
    theta = np.arccos(z)
    return theta, phi


def sh_residual_jacobian(theta, phi, lmax, want_jac=True):
    """Real orthonormal spherical harmonics of even degree 2..lmax.

    Returns r (E,) = sum over points, and if want_jac the tangent Jacobian
    (E, 2m): d/dtheta and (1/sin theta) d/dphi of each harmonic at each point.
    Normalised associated Legendre recurrences (stable to high degree).
    """
    m = theta.size
    x = np.cos(theta)
    s = np.sin(theta)
    rows_val = []
    rows_jt = []
    rows_jp = []
    inv4pi = 1.0 / math.sqrt(4.0 * math.pi)
    # P~_{mu,mu} (orthonormal incl. 1/sqrt(2pi) azimuthal factor, without sqrt2)
    pmm = np.full(m, inv4pi)
    qmm_prev = None  # P~_{mu-1,mu-1}
    for mu in range(0, lmax + 1):
        if mu > 0:
            fac = math.sqrt((2.0 * mu + 1.0) / (2.0 * mu))
            qmm = fac * pmm  # P~_{mu,mu} / sin(theta)
            pmm = qmm * s
        else:
            qmm = None
        # azimuthal factors
        if mu == 0:
            az = [(None, 1.0)]
        else:
            c = math.sqrt(2.0) * np.cos(mu * phi)
            sn = math.sqrt(2.0) * np.sin(mu * phi)
            az = [(c, -mu * sn), (sn, mu * c)]  # (value, d/dphi) pairs
        # l-recurrence on P (and on Q = P/s for mu >= 1)
        p_lm2 = None
        p_lm1 = pmm
        q_lm2 = None
        q_lm1 = qmm
        for l in range(mu, lmax + 1):
            if l == mu:
                p_l, q_l = pmm, qmm
            elif l == mu + 1:
                f = math.sqrt(2.0 * mu + 3.0)
                p_l = f * x * p_lm1
                q_l = f * x * q_lm1 if mu > 0 else None
            else:
                a = math.sqrt((4.0 * l * l - 1.0) / (l * l - mu * mu))
                b = math.sqrt(((l - 1.0) ** 2 - mu * mu) / (4.0 * (l - 1.0) ** 2 - 1.0))
                p_l = a * (x * p_lm1 - b * p_lm2)
                q_l = a * (x * q_lm1 - b * q_lm2) if mu > 0 else None
            if l >= 2 and l % 2 == 0:
                # dP/dtheta
                if want_jac:
                    if l == mu:
                        prev_p, prev_q = 0.0, 0.0
                    else:
                        prev_p, prev_q = p_lm1, q_lm1
                    cl = math.sqrt((2.0 * l + 1.0) * (l * l - mu * mu) / (2.0 * l - 1.0))
                    if mu > 0:
                        dp = l * x * q_l - cl * prev_q
                        pos = q_l  # P/s for the phi derivative
                    else:
                        dp = (l * x * p_l - cl * prev_p) / np.maximum(s, 1e-300)
                        pos = None
                for (v, dv) in az:
                    if v is None:
                        rows_val.append(p_l.sum())
                        if want_jac:
                            rows_jt.append(dp)
                            rows_jp.append(np.zeros(m))
                    else:
                        rows_val.append((p_l * v).sum())
                        if want_jac:
                            rows_jt.append(dp * v)
                            rows_jp.append(pos * dv)
            p_lm2, p_lm1 = p_lm1, p_l
            q_lm2, q_lm1 = q_lm1, q_l
    scale = math.sqrt(4.0 * math.pi) / m
    r = np.array(rows_val) * scale
    if not want_jac:
        return r, None
    J = np.empty((len(rows_val), 2 * m))
    J[:, :m] = np.array(rows_jt)
    J[:, m:] = np.array(rows_jp)
    J *= scale
    return r, J


def solve_design(t, verbose=True, max_iter=200, target=2e-13):
    m = n_free_points(t)
    theta, phi = fibonacci_hemisphere(m)
    if t == 1:
        return np.array([[0.0, 0.0, 1.0]]), 0.0
    lmax = t - 1
    lam = 1e-6
    r, J = sh_residual_jacobian(theta, phi, lmax)
    res = float(np.linalg.norm(r))
    t0 = time.time()
    for it in range(max_iter):
        if res < target:
            break
        A = dsyrk(1.0, J)  # upper triangle of J J^T
        A = np.triu(A) + np.triu(A, 1).T
        diag = np.diag(A).copy()
        accepted = False
        for _ in range(30):
            Al = A + lam * np.diag(diag + 1e-30)
            try:
                cf = cho_factor(Al, lower=False, check_finite=False)
            except np.linalg.LinAlgError:
                lam *= 10.0
                continue
            y = cho_solve(cf, r, check_finite=False)
            d = -(J.T @ y)
            sn = np.sin(theta)
            th_new = theta + d[:m]
            ph_new = phi + d[m:] / np.maximum(sn, 1e-12)
            r_new, _ = sh_residual_jacobian(th_new, ph_new, lmax, want_jac=False)
            res_new = float(np.linalg.norm(r_new))
            if res_new < res:
                theta, phi = th_new, ph_new
                lam = max(lam / 10.0, 1e-15)
                accepted = True
                break
            lam *= 10.0
        if not accepted:
            break
        r, J = sh_residual_jacobian(theta, phi, lmax)
        res = float(np.linalg.norm(r))
        if verbose:
            print(f"  t={t} it={it} res={res:.3e} lam={lam:.1e} ({time.time()-t0:.1f}s)", flush=True)
    pts = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], axis=1)
    pts /= np.linalg.norm(pts, axis=1, keepdims=True)
    return pts, res


def read_store(path):
    out = {}
    if not os.path.exists(path):
        return out
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError("bad t-design store")
    (count,) = struct.unpack_from("<I", data, 8)
    off = 12
    for _ in range(count):
        t, m, _r, res = struct.unpack_from("<IIId", data, off)
        off += 20
        pts = np.frombuffer(data, dtype="<f8", count=3 * m, offset=off).reshape(m, 3).copy()
        off += 24 * m
        out[t] = (pts, res)
    return out


def write_store(path, designs):
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", len(designs)))
        for t in sorted(designs):
            pts, res = designs[t]
            f.write(struct.pack("<IIId", t, pts.shape[0], 0, res))
            f.write(np.ascontiguousarray(pts, dtype="<f8").tobytes())
    os.replace(tmp, path)


def write_reference_dir(store_path, out_dir):
    """Render the store in the reference's directory layout (ssTTT.NNNNN)."""
    designs = read_store(store_path)
    os.makedirs(out_dir, exist_ok=True)
    for t, (pts, _res) in designs.items():
        full = np.concatenate([pts, -pts], axis=0)
        name = os.path.join(out_dir, "ss%03d.%05d" % (t, full.shape[0]))
        with open(name, "w") as f:
            for p in full:
                f.write("%25.16e%25.16e%25.16e\n" % (p[0], p[1], p[2]))
    return out_dir


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tmin", type=int, default=1)
    ap.add_argument("--tmax", type=int, default=141)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "tdesigns.bin"))
    ap.add_argument("--refdir", default=None, help="also write the reference text layout here")
    args = ap.parse_args()
    designs = read_store(args.out)
    for t in range(args.tmin | 1, args.tmax + 1, 2):
        if t in designs and designs[t][1] < 1e-12:
            continue
        t0 = time.time()
        pts, res = solve_design(t, verbose=(t >= 41))
        print(f"t={t} m={pts.shape[0]} residual={res:.3e} time={time.time()-t0:.1f}s", flush=True)
        if res > 1e-12:
            print(f"WARNING: t={t} did not converge", flush=True)
        designs[t] = (pts, res)
        write_store(args.out, designs)
    if args.refdir:
        write_reference_dir(args.out, args.refdir)


if __name__ == "__main__":
    sys.exit(main())
