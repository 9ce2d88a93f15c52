"""The P1 normaliser CF(-i) (heston.rs:86, bates.rs:55-56) as the reference
evaluates it (the oracle's restatement of stable_cf and jump_cf), over the
parameter region where the device kernels take Log CF(-i) = rT without
evaluating it (cf_device.cuh: make_consts) and over the region where they
evaluate it with the reference's sequence:

* regular region (kappa - rho sigma a positive normal number, moderate
  kappa theta / sigma^2, v0 / sigma^2, rT, T and jump terms): the reference's
  Log CF(-i) equals rT to within a few ulps, so the shortcut changes the P1
  integrand by a rounding-level factor only;
* kappa - rho sigma <= 0: the reference's CF(-i) is not finite (every P1
  node is dropped), which the kernels reproduce by taking the reference's
  sequence there."""
import cmath
import math

import numpy as np
import pytest

from oracle import oracle as O


def _draw(rng):
    v0 = rng.uniform(0.001, 0.5)
    kappa = math.exp(rng.uniform(math.log(0.05), math.log(20.0)))
    theta = rng.uniform(0.001, 0.5)
    sigma = rng.uniform(0.05, 3.0)
    rho = rng.uniform(-0.99, 0.99)
    t = math.exp(rng.uniform(math.log(1e-4), math.log(10.0)))
    r = rng.uniform(0.0, 0.1)
    return [v0, kappa, theta, sigma, rho], t, r


def _regular(hp, t, r, jumps=None):
    v0, kappa, theta, sigma, rho = hp
    xr = kappa - rho * sigma
    sig2 = sigma * sigma
    ok = 1e-100 < xr < 1e100 and sig2 > 1e-100 and (kappa * theta) / sig2 < 1e4 and v0 / sig2 * xr < 1e4 \
        and abs(r * t) < 700.0 and t < 1e3
    if jumps is not None:
        lam, mu, sj = jumps
        ok = ok and abs(mu + 0.5 * sj * sj) < 50.0 and abs(lam * t) * math.exp(mu + 0.5 * sj * sj) < 1e4
    return ok


@pytest.mark.parametrize("bates", [False, True])
def test_reference_normaliser_is_exp_rt_in_the_regular_region(bates):
    rng = np.random.default_rng(21 + bates)
    n_reg = n_deg = 0
    for _ in range(4000):
        hp, t, r = _draw(rng)
        jumps = [rng.uniform(0.0, 5.0), rng.uniform(-0.5, 0.3), rng.uniform(0.01, 0.6)] if bates else None
        cf = O.stable_cf(complex(0.0, -1.0), t, r, hp)
        if bates:
            cf = cf * O.jump_cf(complex(0.0, -1.0), t, hp + jumps)  # a full Bates parameter vector
        finite = math.isfinite(cf.real) and math.isfinite(cf.imag) and cf != 0
        xr = hp[1] - hp[3 + 1] * hp[3]
        if _regular(hp, t, r, jumps):
            n_reg += 1
            assert finite
            lg = cmath.log(cf)
            assert abs(lg.real - r * t) <= 4e-16 * max(1.0, abs(r * t)) + 1e-15, (hp, t, r, lg)
            assert abs(lg.imag) <= 1e-15
        if xr <= 0.0:
            n_deg += 1
            assert not finite, (hp, t, r, cf)
    assert n_reg > 2500 and n_deg > 300
