"""CPU checks of the node evaluation's own math functions (csrc/cf_device.cuh):
their polynomial coefficients are the ones csrc/node_math_coeffs.py derives,
and each algorithm, restated in numpy, stays within a few ulps of numpy's
function (the device builds are compared with CUDA's functions by the GPU
tests of ope_selftest_atan2 and ope_selftest_log)."""
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "options-pricing-engine-rs_b200", "csrc")


def _header_coefficients():
    src = open(os.path.join(CSRC, "cf_device.cuh")).read()
    body = src[src.index("double atan2_node("):]
    body = body[:body.index("double r = fma(t * s, p, t);")]
    return [float(v) for v in re.findall(r"(-?\d+\.\d+(?:e-?\d+)?)\)?;", body.split("double p = ", 1)[1])]


def test_coefficients_match_their_generator():
    sys.path.insert(0, CSRC)
    import node_math_coeffs

    c, _ = node_math_coeffs.atan_coefficients()
    want = [float(v) for v in reversed(c)]  # Horner order: highest degree first
    got = _header_coefficients()
    assert got == want, (got, want)


def _atan2_node(y, x, coef):
    ax, ay = np.abs(x), np.abs(y)
    swap = ay > ax
    q = np.where(swap, ax, ay) / np.where(swap, ay, ax)
    big = q > 0.41421356237309503
    t = np.where(big, (q - 1.0) / (q + 1.0), q)
    s = t * t
    p = np.full_like(s, coef[0])
    for cj in coef[1:]:
        p = p * s + cj
    r = t + (t * s) * p
    r = np.where(big, r + 0.78539816339744831, r)
    r = np.where(swap, 1.5707963267948966 - r, r)
    r = np.where(x < 0.0, 3.1415926535897931 - r, r)
    return np.copysign(r, y)


def test_restated_algorithm_within_four_ulp_of_arctan2():
    rng = np.random.default_rng(7)
    n = 1 << 20
    y = rng.choice([-1.0, 1.0], n) * np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-60, 61, n))
    x = rng.choice([-1.0, 1.0], n) * np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-60, 61, n))
    got = _atan2_node(y, x, _header_coefficients())
    ref = np.arctan2(y, x)
    ulp = np.abs(got.view(np.int64) - ref.view(np.int64))
    assert int(ulp.max()) <= 4, int(ulp.max())


def _log_header_coefficients():
    src = open(os.path.join(CSRC, "cf_device.cuh")).read()
    body = src[src.index("double log_node("):]
    body = body[:body.index("const double lm = ")]
    return [float(v) for v in re.findall(r"(-?\d+\.\d+(?:e-?\d+)?)\)?;", body.split("double r = ", 1)[1])]


def test_log_coefficients_match_their_generator():
    sys.path.insert(0, CSRC)
    import node_math_coeffs

    c, _ = node_math_coeffs.log_coefficients()
    assert _log_header_coefficients() == [float(v) for v in reversed(c)]


def _log_node(v, coef):
    bits = v.view(np.int64)
    hi = (bits >> 32).astype(np.int64)
    k = (hi - 0x3FE6A09E) >> 20
    m = (bits - (k << 52)).view(np.float64)
    f = m - 1.0
    s = f / (2.0 + f)
    w = s * s
    r = np.full_like(w, coef[0])
    for cj in coef[1:]:
        r = r * w + cj
    lm = 2.0 * s + (s * w) * r
    kd = k.astype(np.float64)
    return kd * 0.6931471805599453 + (kd * 2.3190468138462996e-17 + lm)


def test_log_restated_algorithm_within_three_ulp_of_numpy():
    rng = np.random.default_rng(11)
    n = 1 << 20
    wide = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-1000, 1001, n))
    near_one = rng.uniform(0.5, 4.0, n)
    for v in (wide, near_one):
        got = _log_node(v, _log_header_coefficients())
        ref = np.log(v)
        ulp = np.abs(got.view(np.int64) - ref.view(np.int64))
        assert int(ulp.max()) <= 3, int(ulp.max())
