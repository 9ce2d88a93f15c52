"""GPU: randomised parity against the oracle over wider ranges than the
benchmark configurations -- vol-of-vol up to 3, correlation up to +-0.99,
mean reversion from 0.05 to 20, Feller violated half the time, expiries from
one day to ten years, strikes from deep in to deep out of the money, jump
intensities up to 5 -- at the reference's tolerance and at 1e-10, one
parameter set per contract.  The bar is the parity bar: 1e-9 S per contract.
Where the reference's own formula gives a non-finite price the device must
too (checked by comparing the finite masks)."""
import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu

S = 100.0


def _draw(rng, n, bates):
    con = np.zeros(n, W.CONTRACT_DTYPE)
    t = np.exp(rng.uniform(np.log(1 / 365), np.log(10.0), n))
    r = rng.uniform(-0.01, 0.08, n)
    q = rng.uniform(0.0, 0.05, n)
    m = rng.uniform(-2.0, 1.2, n) * np.sqrt(np.minimum(t, 1.0))
    con["spot"], con["strike"], con["expiry"] = S, S * np.exp((r - q) * t + m), t
    con["rate"], con["div_yield"], con["vol"] = r, q, 0.2
    con["opt_type"] = rng.integers(0, 2, n)
    p = np.column_stack([rng.uniform(0.005, 0.6, n), np.exp(rng.uniform(np.log(0.05), np.log(20.0), n)),
                         rng.uniform(0.005, 0.6, n), rng.uniform(0.05, 3.0, n), rng.uniform(-0.99, 0.99, n)])
    if bates:
        p = np.column_stack([p, rng.uniform(0.0, 5.0, n), rng.uniform(-0.5, 0.3, n), rng.uniform(0.02, 0.6, n)])
    return con, p


@pytest.mark.parametrize("bates", [False, True])
@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_wide_range_parity(ope, oracle, bates, tol):
    rng = np.random.default_rng(2024 + 7 * bates + int(tol < 1e-9))
    n = 8000
    con, p = _draw(rng, n, bates)
    off = np.arange(n + 1, dtype=np.int64)  # one parameter set (surface) per contract
    got = ope.price_surfaces(ope.MODEL_BATES if bates else ope.MODEL_HESTON, con, off, p, tol=tol)
    ref = oracle.batch_price(con, p, bates, tol, surf_idx=np.arange(n, dtype=np.int32))
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(got), fin)
    err = np.abs(got[fin] - ref[fin])
    worst = int(np.argmax(err))
    print(f"bates={bates} tol={tol}: {fin.sum()} finite of {n}, worst |gpu - oracle| / S = {err.max() / S:.2e}")
    assert err.max() <= 1e-9 * S, (float(err.max()), con[fin][worst], p[fin][worst])


@pytest.mark.parametrize("bates", [False, True])
def test_wide_range_gradient_parity(ope, oracle, bates):
    """The reverse-mode gradient against the oracle's forward-mode AD
    (ad.rs:695-731, 882-895) over the same wide ranges, at the adjoint's bar:
    1e-7 relative plus 1e-9 S absolute per component."""
    rng = np.random.default_rng(77 + bates)
    n = 2000
    con, p = _draw(rng, n, bates)
    off = np.arange(n + 1, dtype=np.int64)
    price, grad = ope.price_gradient_surfaces(ope.MODEL_BATES if bates else ope.MODEL_HESTON, con, off, p, tol=1e-8)
    rp, rg = oracle.batch_price_gradient(con, p, bates, 1e-8, surf_idx=np.arange(n, dtype=np.int32))
    fin = np.all(np.isfinite(rg), axis=1) & np.isfinite(rp)
    assert fin.mean() > 0.99
    lim = 1e-7 * np.abs(rg[fin]) + 1e-9 * S
    ratio = np.abs(grad[fin] - rg[fin]) / lim
    i, k = np.unravel_index(int(np.argmax(ratio)), ratio.shape)
    print(f"bates={bates}: {fin.sum()} of {n}, worst error / bar = {ratio.max():.3g} (component {k})")
    assert ratio.max() <= 1.0, (float(ratio.max()), int(k), con[fin][i], p[fin][i], grad[fin][i], rg[fin][i])


NAMES = ["price", "delta", "gamma", "vega", "theta", "rho", "vanna", "volga"]
# finite-difference amplification of the 1e-9 S price bar in each Greek's formula
AMP = {"price": 1, "delta": 1, "gamma": 4, "vega": 100, "theta": 2 * 365, "rho": 1e4, "vanna": 200, "volga": 2e4}


@pytest.mark.parametrize("bates", [False, True])
def test_wide_range_bump_greeks(ope, oracle, bates):
    """greeks.rs:19-72 (14 pricings per contract) over the wide ranges: 24
    random parameter sets x 64 random contracts each, against the oracle."""
    rng = np.random.default_rng(501 + bates)
    worst = 0.0
    for _ in range(24):
        con, p = _draw(rng, 64, bates)
        got = (ope.batch_bates_greeks if bates else ope.batch_heston_greeks)(con, p[0], tol=1e-10)
        ref = oracle.batch_greeks(con, p[0], bates, tol=1e-10)
        fin = np.all(np.isfinite(ref), axis=1)
        for i, nm in enumerate(NAMES):
            err = np.abs(got[nm][fin] - ref[fin, i]) / (1e-9 * S * AMP[nm])
            worst = max(worst, float(err.max()))
            assert err.max() <= 1.0, (nm, float(err.max()), p[0])
    print(f"bates={bates}: bump Greeks worst error / bar = {worst:.3g}")


@pytest.mark.parametrize("bates", [False, True])
def test_wide_range_ad_greeks(ope, oracle, bates):
    """ad.rs:736-865 over the wide ranges: 16 parameter sets x 32 contracts."""
    rng = np.random.default_rng(601 + bates)
    worst = 0.0
    for _ in range(16):
        con, p = _draw(rng, 32, bates)
        got = ope.batch_greeks_ad(ope.MODEL_BATES if bates else ope.MODEL_HESTON, con, p[0], tol=1e-8)
        ref = np.array([oracle.greeks_ad(c, p[0], bates, 1e-8) for c in con])
        fin = np.all(np.isfinite(ref), axis=1)
        for i, nm in enumerate(NAMES):
            bar = 1e-9 * S * AMP[nm]
            if nm == "vega":
                bar = bar + 1e-7 * np.abs(ref[fin, 3])
            if nm == "volga":
                bar = bar + 1e-7 * 2.0 * (np.abs(ref[fin, 3]) + 1.0) / 0.02
            err = np.abs(got[nm][fin] - ref[fin, i]) / bar
            worst = max(worst, float(err.max()))
            assert err.max() <= 1.0, (nm, float(err.max()), p[0])
    print(f"bates={bates}: AD Greeks worst error / bar = {worst:.3g}")


def test_wide_range_implied_vol(ope, oracle):
    """iv.rs:14-95 on the device over BSM prices of random contracts (vol from
    1 % to 300 %, expiries from a day to ten years), against the oracle: the
    same ok flags where the price carries time value, and the same IVs at the
    vega-scaled bar of the IV tests."""
    rng = np.random.default_rng(701)
    n = 20000
    con, _ = _draw(rng, n, False)
    con["vol"] = np.exp(rng.uniform(np.log(0.01), np.log(3.0), n))
    px = np.array([oracle.bsm_price(c) for c in con])
    got, ok = ope.batch_implied_vol(con, px)
    ref, rok = oracle.batch_implied_vol(con, px)
    eq, er = np.exp(-con["div_yield"] * con["expiry"]), np.exp(-con["rate"] * con["expiry"])
    intrinsic = np.where(con["opt_type"] == 0, np.maximum(S * eq - con["strike"] * er, 0.0),
                         np.maximum(con["strike"] * er - S * eq, 0.0))
    ident = (px - intrinsic) > 1e-9 * S
    assert np.array_equal(ok[ident].astype(bool), rok[ident].astype(bool))
    both = ident & ok.astype(bool) & rok.astype(bool)
    vega = np.array([oracle.bsm_price_and_greeks(oracle.contracts(c["spot"], c["strike"], c["expiry"], c["rate"],
                                                                  c["div_yield"], c["opt_type"], vol=v))[3]
                     for c, v in zip(con[both], ref[both])])
    err = np.abs(got[both] - ref[both]) / (2.5e-10 / np.maximum(vega, 1e-300) + 1e-12)
    print(f"implied vol: {both.sum()} of {n} compared, worst error / bar = {err.max():.3g}")
    assert err.max() <= 1.0


def test_wide_range_calibration(ope, oracle):
    """calibration.rs:433-569 on 12 random Heston surfaces (true parameters over
    wide, Feller-respecting ranges, IV noise of 0.2 vol points, perturbed
    starts): the device LM against the oracle running the same LM with the
    same exact Jacobian (jac_mode=1).  Where both converge they must reach the
    same fit; both must stop for the same reason on most surfaces."""
    rng = np.random.default_rng(901)
    agree = 0
    for k in range(12):
        while True:
            tp = np.array([rng.uniform(0.01, 0.3), rng.uniform(0.3, 8.0), rng.uniform(0.01, 0.3),
                           rng.uniform(0.1, 1.5), rng.uniform(-0.95, 0.5)])
            if 2 * tp[1] * tp[2] > tp[3] ** 2:
                break
        rows = []
        for t in (0.1, 0.5, 1.0, 2.0):
            for m in (-0.4, -0.2, -0.1, 0.0, 0.1, 0.2, 0.3):
                rows.append((S, S * np.exp(m), t, 0.02, 0.01, 0.2, 0 if m >= 0 else 1, 0))
        con = np.array(rows, dtype=W.CONTRACT_DTYPE)
        px = oracle.batch_price(con, tp, False, 1e-10)
        iv, ok = oracle.batch_implied_vol(con, px)
        con, iv = con[ok.astype(bool)], iv[ok.astype(bool)] + rng.normal(0.0, 0.002, ok.sum())
        p0 = tp * rng.uniform(0.8, 1.2, 5)
        p0[3] = min(p0[3], 0.95 * np.sqrt(2 * p0[1] * p0[2]))
        g = ope.calibrate_heston(con, iv, p0)
        o = oracle.calibrate_ex(5, con, iv, p0, jac_mode=1)
        if g["converged"] and o["converged"]:
            assert abs(g["rmse"] - o["rmse"]) < 1e-9, (k, g["rmse"], o["rmse"])
            assert np.allclose(g["params"][:5], o["params"][:5], rtol=1e-5, atol=1e-8), (k, g["params"][:5],
                                                                                        o["params"][:5])
        agree += int(g["converged"] == o["converged"] and g["early_stopped"] == o["early_stopped"])
    print(f"calibration: {agree} of 12 surfaces stop the same way")
    assert agree >= 10


@pytest.mark.parametrize("bates", [False, True])
def test_extreme_inputs_parity(ope, oracle, bates):
    """Corners: tolerance 1e-12 (the 200-panel cap binds often), expiries down
    to 1e-4 years, log-moneyness out to +-4, zero rates, near-zero v0 and
    theta.  Same finiteness and the 1e-9 S bar."""
    rng = np.random.default_rng(1301 + bates)
    n = 4000
    con, p = _draw(rng, n, bates)
    t = np.exp(rng.uniform(np.log(1e-4), np.log(10.0), n))
    con["expiry"] = t
    con["strike"] = S * np.exp(rng.uniform(-4.0, 4.0, n))
    zero = rng.random(n) < 0.2
    con["rate"][zero], con["div_yield"][zero] = 0.0, 0.0
    small = rng.random(n) < 0.2
    p[small, 0] = rng.uniform(1e-6, 1e-4, small.sum())
    p[small, 2] = rng.uniform(1e-6, 1e-4, small.sum())
    off = np.arange(n + 1, dtype=np.int64)
    got = ope.price_surfaces(ope.MODEL_BATES if bates else ope.MODEL_HESTON, con, off, p, tol=1e-12)
    ref = oracle.batch_price(con, p, bates, 1e-12, surf_idx=np.arange(n, dtype=np.int32))
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(got), fin)
    err = np.abs(got[fin] - ref[fin])
    print(f"bates={bates} extreme: {fin.sum()} finite of {n}, worst |gpu - oracle| / S = {err.max() / S:.2e}")
    assert err.max() <= 1e-9 * S
