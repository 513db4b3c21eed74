"""The FMA-pipe sine/cosine of the structure-factor kernel (CPU).

The constants compiled into kernels.cuh must be the ones fit_sincos.py fits,
and the kernel's FP32 operation sequence (emulated exactly: each FMA is an
exact product plus one rounding) must stay within 2e-7 of sin/cos on the
phase range the kernel sees (|theta| <= 30 rad), about a third of the error
of the MUFU sin.approx/cos.approx it stands in for.
"""
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gauss-legendre-spherical-t_b200", "csrc")
sys.path.insert(0, CSRC)
import fit_sincos  # noqa: E402

sys.path.pop(0)


def _header_constants():
    text = open(os.path.join(CSRC, "kernels.cuh")).read()
    vals = dict((m.group(1), float(m.group(2)))
                for m in re.finditer(r"\b(k(?:Sin\d|Cos\d|PiHi|PiLo|InvPi|RoundMagic))\s*=\s*([-+0-9.eE]+)f", text))
    return vals


def test_header_constants_are_the_fitted_ones():
    h = _header_constants()
    sc, cc = fit_sincos.coefficients()
    assert [np.float32(h["kSin%d" % i]) for i in range(1, 5)] == list(sc)
    assert [np.float32(h["kCos%d" % i]) for i in range(5)] == list(cc)
    assert np.float32(h["kPiHi"]) == np.float32(3.140625)
    assert np.float32(h["kPiLo"]) == np.float32(np.pi - 3.140625)
    assert np.float32(h["kInvPi"]) == np.float32(1.0 / np.pi)
    assert h["kRoundMagic"] == 12582912.0


def test_error_bound():
    sc, cc = fit_sincos.coefficients()
    es, ec = fit_sincos.max_error(sc, cc, bound=30.0, n=400001)
    assert es <= 2e-7 and ec <= 2e-7, (es, ec)
    # far outside the usual phase range the reduction still holds
    es, ec = fit_sincos.max_error(sc, cc, bound=400.0, n=400001)
    assert es <= 1e-6 and ec <= 1e-6, (es, ec)
    # sign handling at the reduction boundaries: theta = (m + 1/2) pi
    th = (np.arange(-9, 9) + 0.5) * np.pi
    s, c = fit_sincos.emulate(th, sc, cc)
    assert np.allclose(s, np.sin(th.astype(np.float32).astype(np.float64)), atol=3e-7)
    assert np.allclose(c, np.cos(th.astype(np.float32).astype(np.float64)), atol=3e-7)
