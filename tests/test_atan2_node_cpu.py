"""CPU checks of the node evaluation's own atan2 (atan2_node in
csrc/cf_device.cuh): its polynomial coefficients are the ones
csrc/atan_coeffs.py derives, and the algorithm, restated in numpy, stays
within a few ulps of numpy's arctan2 (the device build is compared with
CUDA's atan2 by the GPU test of ope_selftest_atan2)."""
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
    import atan_coeffs

    c, _ = atan_coeffs.coefficients()
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
