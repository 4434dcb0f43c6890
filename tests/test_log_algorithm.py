"""CPU checks of the fused FP64 kernels' own logarithm (pf_log in
pf3d_device.cuh), beside the device test in test_math_log_gpu.py:

* the seven polynomial coefficients in the header are the ones
  csrc/log_coeffs.py derives (Chebyshev interpolant of the atanh tail), and
  the split of ln2 has an exact product head;
* a step-by-step restatement of pf_log's arithmetic (high-word reduction,
  compensated quotient, Horner, final sums; every fma exact-then-rounded)
  stays within 1 ulp of the exact logarithm when the reciprocal it starts
  from is off by up to one ulp, as the device's may be.
"""
import math
import os
import re
import struct
from fractions import Fraction

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "phase-field-project-3d_b200", "csrc")
LN2_HI = 0.6931467056274414
LN2_LO = 4.7493250390316726e-07


def _header_coeffs():
    src = open(os.path.join(CSRC, "pf3d_device.cuh")).read()
    body = src[src.index("__device__ __forceinline__ double pf_log(double x)"):]
    body = body[:body.index("\n}\n")]
    first = re.search(r"double p = ([0-9.e+-]+);", body).group(1)
    rest = re.findall(r"p = __fma_rn\(p, z, ([0-9.e+-]+)\);", body)
    return [float(first)] + [float(c) for c in rest]


def test_header_coefficients_match_generator():
    pytest.importorskip("mpmath")
    import sys
    sys.path.insert(0, CSRC)
    try:
        import log_coeffs
    finally:
        sys.path.remove(CSRC)
    coeffs, worst = log_coeffs.coefficients(grid=1000)
    assert _header_coeffs() == coeffs
    assert worst * float(log_coeffs.Z_MAX) < 1e-17


def test_ln2_split():
    hi_bits = struct.unpack("<Q", struct.pack("<d", LN2_HI))[0]
    assert hi_bits & 0xFFFFFFFF == 0            # k * ln2_hi exact for |k| < 2^21
    assert hi_bits == 0x3FE62E4200000000
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 40
    assert abs(mp.mpf(LN2_HI) + mp.mpf(LN2_LO) - mp.log(2)) < mp.mpf(2) ** -75


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _restated_log(x, rcp_ulps, coeffs):
    b = struct.unpack("<Q", struct.pack("<d", x))[0]
    hi, lo = b >> 32, b & 0xFFFFFFFF
    hi += 0x3FF00000 - 0x3FE6A09E
    k = (hi >> 20) - 0x3FF
    m = struct.unpack("<d", struct.pack("<Q", (((hi & 0x000FFFFF) + 0x3FE6A09E) << 32) | lo))[0]
    f = m - 1.0
    d = 2.0 + f
    derr = f - (d - 2.0)
    rc = 1.0 / d
    for _ in range(abs(rcp_ulps)):                # a reciprocal off by up to one ulp
        rc = math.nextafter(rc, math.inf if rcp_ulps > 0 else -math.inf)
    s = f * rc
    e = _fma(-s, derr, _fma(-s, d, f))
    sl = e * rc
    z = s * s
    p = coeffs[0]
    for c in coeffs[1:]:
        p = _fma(p, z, c)
    t = 2.0 * s
    lo_sum = _fma(t * z, p, sl + sl)
    kd = float(k)
    return _fma(kd, LN2_HI, _fma(kd, LN2_LO, lo_sum) + t)


def test_restated_log_within_one_ulp():
    coeffs = _header_coeffs()
    rng = np.random.default_rng(11)
    xs = np.concatenate([
        np.exp(rng.uniform(-700.0, 700.0, 600)),
        1.0 + rng.uniform(-0.3, 0.45, 600),
        rng.uniform(0.3, 0.75, 400),
        np.sqrt(2.0) * (1.0 + rng.uniform(-1e-6, 1e-6, 200)),
        np.sqrt(0.5) * (1.0 + rng.uniform(-1e-6, 1e-6, 200)),
        10.0 ** rng.uniform(-6.0, 2.0, 400),
        [1.0, 2.0, 0.5, np.finfo(np.float64).tiny, np.finfo(np.float64).max],
    ])
    worst = 0.0
    for q, x in enumerate(xs):
        x = float(x)
        y = _restated_log(x, (-1, 0, 1)[q % 3], coeffs)
        ref = np.log(np.longdouble(x))
        ulp = np.spacing(abs(np.float64(ref)))
        worst = max(worst, float(abs(np.longdouble(y) - ref)) / float(ulp) if ulp else 0.0)
    assert worst <= 1.0, worst
    assert _restated_log(1.0, 0, coeffs) == 0.0
