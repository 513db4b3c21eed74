"""Fit the coefficients of the FMA-pipe sine/cosine in kernels.cuh.

    sin r = r + r^3 (S1 + S2 r^2 + S3 r^4 + S4 r^6)
    cos r = C0 + C1 r^2 + C2 r^4 + C3 r^6 + C4 r^8,        |r| <= pi/2

Each is a polynomial in x = r^2 on [0, (pi/2)^2], fitted to sin(r)/r and
cos(r) by least squares on Chebyshev points with Lawson reweighting (the
weights grow where the error is largest, which drives the fit toward the
minimax one), then rounded to FP32.  ``emulate`` evaluates the kernel's
sequence of FP32 operations (FMAs as exact products and one rounding) so the
printed error bound is the one of the device code, range reduction included.

    python fit_sincos.py
"""
import numpy as np

F32 = np.float32
HALF_PI = np.pi / 2


def fit(fun, degree, n=4000, iterations=60):
    t = np.cos(np.pi * (np.arange(n) + 0.5) / n)
    r = np.concatenate([HALF_PI * (t + 1) / 2, [HALF_PI]])
    x = r * r
    y = fun(r)
    a = np.vstack([x ** k for k in range(degree + 1)]).T
    w = np.ones_like(x)
    c = None
    for _ in range(iterations):
        sw = np.sqrt(w)
        c, *_ = np.linalg.lstsq(a * sw[:, None], y * sw, rcond=None)
        e = np.abs(a @ c - y)
        w = w * (e / e.max() + 1e-12)
        w /= w.sum()
    return c.astype(F32)


def coefficients():
    s = fit(lambda r: np.sin(r) / r, 4)   # 1, S1..S4
    c = fit(np.cos, 4)                    # C0..C4
    return s[1:], c


def _fma(a, b, c):
    return F32(np.float64(a) * np.float64(b) + np.float64(c))


def emulate(theta, sin_coef, cos_coef):
    """FP32 sin/cos of theta by the kernel's steps; returns (sin, cos)."""
    theta = np.asarray(theta, dtype=F32)
    inv_pi, magic = F32(1.0 / np.pi), F32(12582912.0)
    pi_hi = F32(3.140625)
    pi_lo = F32(np.pi - 3.140625)
    t = _fma(theta, inv_pi, magic)
    n = F32(t - magic)
    r = _fma(-n, pi_hi, theta)
    r = _fma(-n, pi_lo, r)
    r2 = F32(r * r)
    s1, s2, s3, s4 = sin_coef
    p = _fma(s4, r2, s3)
    p = _fma(p, r2, s2)
    p = _fma(p, r2, s1)
    s = _fma(F32(p * r2), r, r)
    c0, c1, c2, c3, c4 = cos_coef
    q = _fma(c4, r2, c3)
    q = _fma(q, r2, c2)
    q = _fma(q, r2, c1)
    c = _fma(q, r2, c0)
    sign = np.where((t.view(np.int32) & 1) == 1, F32(-1), F32(1))
    return s * sign, c * sign


def max_error(sin_coef, cos_coef, bound=30.0, n=2000001):
    th = np.linspace(-bound, bound, n).astype(F32)
    s, c = emulate(th, sin_coef, cos_coef)
    ref = th.astype(np.float64)
    return (float(np.abs(s - np.sin(ref)).max()), float(np.abs(c - np.cos(ref)).max()))


if __name__ == "__main__":
    sc, cc = coefficients()
    print("sin:", ", ".join(repr(float(v)) for v in sc))
    print("cos:", ", ".join(repr(float(v)) for v in cc))
    print("max abs error on |theta| <= 30: sin %.2e, cos %.2e" % max_error(sc, cc))
