"""GPU test of the fused FP64 kernels' own logarithm (pf_math_log).

The fast form evaluates log(CL/(1-CL)) and the log| . | of the solute
node with an atanh series after argument reduction instead of CUDA's log.
This holds it to the exact logarithm (x86 long double, 64-bit mantissa, as
the reference value) within 1 ulp of the double result over positive normal
and subnormal arguments, to CUDA's own log within 2 ulp, and checks the
special arguments (0, -0, negatives, +inf, NaN) give IEEE log's results.
"""
import numpy as np
import pytest

import pf3d

pytestmark = pytest.mark.gpu


def _ulps(y, ref):
    ref64 = ref.astype(np.float64)
    return np.abs((y.astype(np.longdouble) - ref) / np.spacing(np.abs(ref64)).astype(np.longdouble)).astype(np.float64)


def _args():
    rng = np.random.default_rng(2024)
    parts = [
        np.exp(rng.uniform(-700.0, 700.0, 200_000)),          # whole normal range
        1.0 + rng.uniform(-0.3, 0.45, 200_000),                # k = 0 and the reduction edges
        rng.uniform(0.3, 0.75, 100_000),                       # k = -1 where |result| is smallest
        np.sqrt(2.0) * (1.0 + rng.uniform(-1e-6, 1e-6, 50_000)),
        np.sqrt(0.5) * (1.0 + rng.uniform(-1e-6, 1e-6, 50_000)),
        1.0 + rng.uniform(-1e-9, 1e-9, 50_000),                # log near 0
        10.0 ** rng.uniform(-6.0, 2.0, 100_000),               # the kernels' ratios CL/(1-CL)
        rng.uniform(1e-310, 2.2e-308, 10_000),                 # subnormals
        np.array([np.finfo(np.float64).tiny, np.finfo(np.float64).max, 1.0, 2.0, 0.5, 5e-324]),
    ]
    return np.concatenate(parts)


def test_own_log_within_one_ulp(gpu):
    x = _args()
    own, lib = pf3d.math_log(x)
    ref = np.log(x.astype(np.longdouble))
    e_own = _ulps(own, ref)
    e_lib = _ulps(lib, ref)
    assert np.isfinite(own).all()
    assert e_own.max() <= 1.0, (e_own.max(), x[np.argmax(e_own)])
    assert (np.abs(own - lib) <= 2.0 * np.spacing(np.abs(lib))).all()
    assert e_own.mean() < 0.5 and e_lib.max() <= 1.0
    assert (own == 0.0)[x == 1.0].all()


def test_own_log_special_arguments(gpu):
    x = np.array([0.0, -0.0, -1.0, -np.inf, np.inf, np.nan, -5e-324])
    own, lib = pf3d.math_log(x)
    assert own[0] == -np.inf and own[1] == -np.inf
    assert np.isnan(own[2]) and np.isnan(own[3]) and np.isnan(own[5]) and np.isnan(own[6])
    assert own[4] == np.inf
    np.testing.assert_array_equal(np.isnan(own), np.isnan(lib))
    np.testing.assert_array_equal(own[~np.isnan(own)], lib[~np.isnan(lib)])
