"""CPU: pin the oracle before trusting it.

The reference (Rust) cannot be built in this environment, so the oracle is
pinned by (a) every invariant the reference's own tests assert on this path,
re-run here against the oracle with the reference's tolerances, and (b)
independent known answers in tests/golden/ (mpmath principal square roots,
mpmath high-precision Gil-Pelaez prices, and the oracle's own committed
fixtures so that later edits cannot drift silently).
"""
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

H_REF = [0.04, 2.0, 0.04, 0.3, -0.7]    # heston.rs:236-239
B_REF = H_REF + [0.5, -0.1, 0.15]       # bates.rs:94-96


# ---- heston.rs:255-307 fast_csqrt_matches_builtin --------------------------
def test_fast_csqrt_matches_principal_sqrt(oracle):
    with open(os.path.join(GOLD, "csqrt_sweep.json")) as f:
        pts = json.load(f)
    assert len(pts) > 250
    worst = 0.0
    axis = {(4.0, 0.0), (-4.0, 0.0), (0.0, 4.0), (0.0, -4.0), (0.0, 0.0)}
    for re, im, sre, sim in pts:
        got = oracle.fast_csqrt(complex(re, im))
        exp = complex(float(sre), float(sim))
        if (re, im) in axis:
            assert abs(got - exp) < 1e-12, (re, im, got, exp)
        else:
            err = abs(got - exp) / max(abs(exp), 1e-300)
            worst = max(worst, err)
            assert err < 1e-9, (re, im, got, exp)
    # the branch-cut sign convention on the exact negative real axis (heston.rs:161-162)
    assert oracle.fast_csqrt(complex(-4.0, -0.0)) == complex(0.0, -2.0)
    assert worst < 1e-15


# ---- independent known answers ---------------------------------------------
def test_oracle_matches_mpmath_known_answers(oracle):
    path = os.path.join(GOLD, "mpmath_prices.json")
    if not os.path.exists(path):
        pytest.skip("mpmath fixtures not generated")
    with open(path) as f:
        cases = json.load(f)
    assert len(cases) >= 40
    worst = 0.0
    for c in cases:
        p = c["params"]
        fn = oracle.bates_price if len(p) == 8 else oracle.heston_price
        v = fn(c["spot"], c["strike"], c["expiry"], c["rate"], c["div_yield"], p, c["opt_type"], 1e-10)
        err = abs(v - float(c["price"]))
        worst = max(worst, err)
        assert err < 1e-8, (c, v)
    assert worst < 1e-8


def test_oracle_fixtures_unchanged(oracle):
    from ope_b200 import workloads as W

    w = W.c1()
    with open(os.path.join(GOLD, "oracle_c1.json")) as f:
        g = json.load(f)
    px = oracle.batch_price(w.contracts, w.params, False, g["tol"])
    gold = np.array([float.fromhex(h) for h in g["price"]])
    assert np.array_equal(px, gold)
    with open(os.path.join(GOLD, "oracle_bates_grid.json")) as f:
        rows = json.load(f)
    for r in rows:
        v = oracle.bates_price(100.0, r["strike"], r["expiry"], 0.03, 0.0, r["params"], 0, 1e-10)
        assert v == float.fromhex(r["price"])


def test_oracle_corner_fixture_unchanged(oracle):
    """The corner contracts of corner_cap_contracts.json (tol 1e-12, both
    integrals at the 200-panel cap): the oracle's prices and bisection counts
    are the committed ones, bit for bit."""
    from ope_b200 import workloads as W

    with open(os.path.join(GOLD, "corner_cap_contracts.json")) as f:
        d = json.load(f)
    for e in d["contracts"]:
        c = np.zeros(1, W.CONTRACT_DTYPE)
        for k, v in e["contract"].items():
            c[k] = float.fromhex(v)
        c["opt_type"] = e["opt_type"]
        p = np.array([[float.fromhex(x) for x in e["params"]]])
        px, nb = oracle.batch_price(c, p, bool(e["bates"]), d["tol"], stats=True)
        assert px[0] == float.fromhex(e["oracle_price"])
        assert list(nb) == e["oracle_bisections"]


def _ref_inputs():
    from ope_b200 import workloads as W

    rows = []
    with open(os.path.join(GOLD, "ref_inputs.txt")) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            lhs, rhs = line.split(";")
            model, *p = lhs.split()
            c = rhs.split()
            con = np.zeros(1, W.CONTRACT_DTYPE)
            for k, v in zip(("spot", "strike", "expiry", "rate", "div_yield"), c[:5]):
                con[k] = float(v)
            con["opt_type"] = 1 if c[5] == "put" else 0
            rows.append((model == "bates", np.array([[float(x) for x in p]]), con))
    return rows


def test_reference_pin_inputs_price_on_the_oracle(oracle):
    """The contracts of ref_inputs.txt (the pin against the reference crate's
    own outputs, oracle/ref_golden/) parse and price on the oracle."""
    rows = _ref_inputs()
    assert len(rows) == 120 + 256 + 12
    for bates, p, c in rows[::37]:
        assert np.isfinite(oracle.batch_price(c, p, bates, oracle.REF_TOL)[0])


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "ref_prices.txt")),
                    reason="no reference outputs: tests/golden/ref_prices.txt is written by "
                           "oracle/ref_golden/make_ref_golden.sh where cargo exists")
def test_oracle_equals_the_reference_crate(oracle):
    """Pinned by the reference itself: the oracle's prices at the reference's
    tolerance equal the reference crate's (heston_price / bates_price) bit for
    bit on every contract of ref_inputs.txt."""
    with open(os.path.join(GOLD, "ref_prices.txt")) as f:
        ref = [float(x) for x in f.read().split()]
    rows = _ref_inputs()
    assert len(ref) == len(rows)
    for (bates, p, c), r in zip(rows, ref):
        assert oracle.batch_price(c, p, bates, oracle.REF_TOL)[0] == r


def test_oracle_trace_replays_its_own_quadrature(oracle):
    """The oracle's step trace of adaptive_gk (heston.rs:193-212) is the
    quadrature it runs: its last total is the integral, its step count is one
    more than the bisection count, and replaying its choices rebuilds a panel
    list whose K values sum to that total."""
    import qag_trace as Q
    from ope_b200 import workloads as W

    w = W.c3(n=512, per_surface=256)
    si = w.surf_idx()
    for i in (0, 7, 300):
        nb = oracle.batch_price(w.contracts[i:i + 1], w.params[si[i]:si[i] + 1], True, w.tol, stats=True)[1]
        for which in (0, 1):
            tr, integral = oracle.trace_integral(w.contracts[i], w.params[si[i]], True, which, w.tol)
            assert len(tr) == nb[which] + 1 and tr[-1, Q.TOTAL] == integral
            live = Q.panels_before(tr, len(tr))
            assert len(live) == len(tr)
            assert abs(sum(k for k, _, _ in live.values()) - integral) <= 1e-12 * max(1.0, abs(integral))


# ---- heston.rs tests --------------------------------------------------------
def test_put_call_parity(oracle):  # heston.rs:309-316
    call = oracle.heston_price(100.0, 100.0, 0.5, 0.03, 0.0, H_REF, 0)
    put = oracle.heston_price(100.0, 100.0, 0.5, 0.03, 0.0, H_REF, 1)
    assert abs(call - put - (100.0 - 100.0 * math.exp(-0.03 * 0.5))) < 0.01


def test_price_sanity(oracle):  # heston.rs:318-327
    call = oracle.heston_price(100.0, 100.0, 1.0, 0.05, 0.0, H_REF, 0)
    put = oracle.heston_price(100.0, 100.0, 1.0, 0.05, 0.0, H_REF, 1)
    assert abs(call - put - 100.0 + 100.0 * math.exp(-0.05)) < 0.05 and call >= 0.0


def test_feller(oracle):  # heston.rs:329-332, types.rs:60-62
    v0, k, th, s, r = H_REF
    assert 2 * k * th > s * s


def _check_arbitrage(price_fn, sets):
    s, r, q = 100.0, 0.03, 0.0
    for p in sets:
        for t in (0.02, 0.1, 0.25, 0.5, 1.0, 2.0):
            cap = s * math.exp(-q * t)
            prev = math.inf
            for k in (70.0, 85.0, 100.0, 115.0, 130.0, 150.0, 200.0):
                c = price_fn(s, k, t, r, q, p, 0)
                intrinsic = max(s * math.exp(-q * t) - k * math.exp(-r * t), 0.0)
                assert c >= intrinsic - 1e-4 and c <= cap + 1e-4 and c <= prev + 1e-4, (p, t, k, c)
                prev = c


def test_no_static_arbitrage_heston(oracle):  # heston.rs:382-406
    _check_arbitrage(oracle.heston_price, [[0.04, 2.0, 0.04, 0.3, -0.7], [0.09, 1.0, 0.09, 0.8, -0.5],
                                           [0.04, 0.5, 0.04, 0.5, -0.7]])


def test_no_static_arbitrage_bates(oracle):  # bates.rs:147-173
    _check_arbitrage(oracle.bates_price, [[0.04, 2.0, 0.04, 0.3, -0.7, 0.5, -0.1, 0.15],
                                          [0.09, 1.0, 0.09, 0.8, -0.5, 1.0, -0.2, 0.25]])


def test_zero_vol_of_vol_matches_bsm(oracle):  # heston.rs:411-427
    p = [0.04, 1.0, 0.04, 1e-4, 0.0]
    for t in (0.25, 1.0, 2.0):
        for k in (70.0, 85.0, 100.0, 115.0, 130.0):
            h = oracle.heston_price(100.0, k, t, 0.03, 0.0, p, 0)
            b = oracle.bsm_price(oracle.contracts(100.0, k, t, 0.03, 0.0, 0, vol=0.2))
            assert abs(h - b) < 0.02


def test_greeks_signs(oracle):  # heston.rs:334-350, bates.rs:117-131
    for bates, p in ((False, H_REF), (True, B_REF)):
        c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, [0, 1])
        g = oracle.batch_greeks(c, p, bates)
        assert 0 < g[0, 1] < 1 and g[0, 2] > 0 and g[0, 3] > 0 and g[0, 5] > 0
        assert -1 < g[1, 1] < 0 and g[1, 2] > 0


def test_delta_close_to_bsm(oracle):  # heston.rs:358-377
    p = [0.04, 0.1, 0.04, 0.01, 0.0]
    c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 0, vol=0.2)
    h = oracle.batch_greeks(c, p, False)[0]
    b = oracle.bsm_price_and_greeks(c)
    assert abs(h[1] - b[1]) < 0.01
    damp = (1.0 - math.exp(-p[1])) / p[1]
    assert abs(h[3] - b[3] * damp) < 0.5


# ---- bates.rs tests ---------------------------------------------------------
def test_bates_recovers_heston_no_jumps(oracle):  # bates.rs:98-106
    b = oracle.bates_price(100.0, 100.0, 1.0, 0.05, 0.0, H_REF + [0.0, 0.0, 1e-8], 0)
    h = oracle.heston_price(100.0, 100.0, 1.0, 0.05, 0.0, H_REF, 0)
    assert abs(b - h) < 0.02


def test_bates_put_call_parity(oracle):  # bates.rs:108-115
    call = oracle.bates_price(100.0, 100.0, 0.5, 0.03, 0.0, B_REF, 0)
    put = oracle.bates_price(100.0, 100.0, 0.5, 0.03, 0.0, B_REF, 1)
    assert abs(call - put - (100.0 - 100.0 * math.exp(-0.03 * 0.5))) < 0.02


def test_bates_greeks_match_heston_no_jumps(oracle):  # bates.rs:134-142
    c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 0)
    b = oracle.batch_greeks(c, H_REF + [0.0, 0.0, 1e-8], True)[0]
    h = oracle.batch_greeks(c, H_REF, False)[0]
    assert abs(b[1] - h[1]) < 0.01 and abs(b[3] - h[3]) < 1.0


# ---- batch.rs tests ---------------------------------------------------------
def _chain(oracle, n):
    return oracle.contracts(100.0, 80.0 + 2.0 * np.arange(n), 0.5, 0.03, 0.0, 0, vol=0.2)


def test_batch_greeks_match_scalar(oracle):  # batch.rs:270-306
    c = _chain(oracle, 15)
    for bates, p in ((False, H_REF), (True, B_REF)):
        g = oracle.batch_greeks(c, p, bates)
        for i in range(c.size):
            s = oracle.batch_greeks(c[i:i + 1], p, bates, nthreads=1)[0]
            assert np.all(np.abs(g[i] - s) < 1e-12)


def test_batch_price_matches_batch_greeks(oracle):  # batch.rs:310-319
    c = _chain(oracle, 12)
    px = oracle.batch_price(c, np.array([H_REF]), False)
    g = oracle.batch_greeks(c, H_REF, False)
    assert np.all(np.abs(px - g[:, 0]) < 1e-12)


# ---- ad.rs tests --------------------------------------------------------------
def test_ad_price_matches_standard(oracle):  # ad.rs:1365-1371
    c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 0)
    ad = oracle.greeks_ad(c, H_REF, False)
    std = oracle.heston_price(100.0, 100.0, 1.0, 0.05, 0.0, H_REF, 0)
    assert abs(ad[0] - std) < 1e-10


def test_ad_price_matches_standard_across_wings(oracle):  # ad.rs:1394-1408, 922-939
    for t in (0.02, 0.1, 0.5, 1.0, 2.0):
        for k in (70.0, 85.0, 100.0, 115.0, 130.0):
            pv, _ = oracle.forward_pass(100.0, k, t, 0.05, 0.0, H_REF, 0, 0)
            assert abs(pv - oracle.heston_price(100.0, k, t, 0.05, 0.0, H_REF, 0)) < 1e-6
            pv, _ = oracle.forward_pass(100.0, k, t, 0.05, 0.0, H_REF, 0, 0, jump=(0.5, -0.1, 0.15))
            assert abs(pv - oracle.bates_price(100.0, k, t, 0.05, 0.0, B_REF, 0)) < 1e-6


def test_ad_vega_close_to_bump(oracle):  # ad.rs:1412-1419, 941-953
    c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 0)
    for bates, p in ((False, H_REF), (True, B_REF)):
        ad = oracle.greeks_ad(c, p, bates)
        bump = oracle.batch_greeks(c, p, bates)[0]
        assert abs(ad[3] - bump[3]) / abs(bump[3]) < 0.01


def test_bates_ad_matches_heston_ad_when_jumps_off(oracle):  # ad.rs:913-921
    c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 0)
    h = oracle.greeks_ad(c, H_REF, False)
    b = oracle.greeks_ad(c, H_REF + [0.0, 0.0, 1e-8], True)
    assert abs(h[0] - b[0]) < 1e-6 and abs(h[3] - b[3]) < 1e-4


def test_jump_sensitivities_match_fd(oracle):  # ad.rs:982-1011
    lam, mu, sj = 0.5, -0.1, 0.15
    s, k, t, r, q = 100.0, 100.0, 1.0, 0.05, 0.0

    def price_at(l_, m_, s_):
        return oracle.bates_price(s, k, t, r, q, H_REF + [l_, m_, s_], 0)

    h = 1e-5
    fd = [(price_at(lam + h, mu, sj) - price_at(lam - h, mu, sj)) / (2 * h),
          (price_at(lam, mu + h, sj) - price_at(lam, mu - h, sj)) / (2 * h),
          (price_at(lam, mu, sj + h) - price_at(lam, mu, sj - h)) / (2 * h)]
    for a in range(3):
        pv, d = oracle.forward_pass(s, k, t, r, q, H_REF, 0, -1, jump=(lam, mu, sj), jump_active=a)
        assert abs(d - fd[a]) / max(abs(fd[a]), 1e-8) < 1e-3, (a, d, fd[a])
        assert abs(pv - price_at(lam, mu, sj)) < 1e-6  # ad.rs:960-972
    _, dmu = oracle.forward_pass(s, k, t, r, q, H_REF, 0, -1, jump=(lam, mu, sj), jump_active=1)
    assert dmu < 0.0  # ad.rs:1022-1027


# ---- math.rs / iv.rs / bsm.rs ----------------------------------------------
def test_ncdf_tail_precision(oracle):  # math.rs:65-76
    for x, e in ((-4.0, 3.167124183311998e-5), (-5.0, 2.866515718791939e-7), (-6.0, 9.865876449133282e-10)):
        assert abs(oracle.ncdf(x) - e) / e < 5e-10
    assert abs(oracle.ncdf(0.0) - 0.5) < 1e-15 and oracle.ncdf(-10.0) < 1e-23


def test_ncdf_inv_roundtrip(oracle):  # math.rs:78-84
    for p in (0.01, 0.1, 0.5, 0.9, 0.99):
        assert abs(oracle.ncdf(oracle.ncdf_inv(p)) - p) < 1e-6


@pytest.mark.parametrize("vol,ot", [(0.2, 0), (0.2, 1), (0.3, 0), (0.05, 0)])
def test_iv_roundtrip(oracle, vol, ot):  # iv.rs:111-124
    c = oracle.contracts(100.0, 100.0, 0.5, 0.03, 0.0, ot, vol=vol)
    px = oracle.bsm_price(c)
    iv = oracle.implied_vol(c, px)
    assert iv is not None and abs(iv - vol) < 1e-7
    assert oracle.implied_vol(c, -1.0) is None  # iv.rs:126-129


def test_bsm_call_put_parity(oracle):  # bsm.rs:234-241
    c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 0, vol=0.2)
    p = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 1, vol=0.2)
    assert abs(oracle.bsm_price(c) - oracle.bsm_price(p) - (100.0 - 100.0 * math.exp(-0.05))) < 1e-10


# ---- calibration.rs ---------------------------------------------------------
def _quotes(oracle, p, bates=False):  # calibration.rs:980-1018
    rows, ivs = [], []
    for t in (0.25, 0.5, 1.0):
        for k in (80.0, 90.0, 95.0, 100.0, 105.0, 110.0, 120.0):
            ot = 0 if k >= 100.0 else 1
            fn = oracle.bates_price if bates else oracle.heston_price
            px = fn(100.0, k, t, 0.03, 0.0, p, ot)
            c = oracle.contracts(100.0, k, t, 0.03, 0.0, ot, vol=0.2)
            iv = oracle.implied_vol(c, px)
            if iv is not None and 0.01 < iv < 2.0:
                rows.append(c[0])
                ivs.append(iv)
    return np.array(rows), np.array(ivs)


def test_calibration_recovers_params(oracle):  # calibration.rs:1020-1038, 1040-1050
    true_p = [0.04, 2.0, 0.04, 0.3, -0.5]
    con, iv = _quotes(oracle, true_p)
    res = oracle.calibrate(5, con, iv, [0.05, 1.5, 0.05, 0.4, -0.3])
    assert res["converged"] and res["rmse"] < 0.005
    p = res["params"][:5]
    assert abs(p[0] - 0.04) < 0.005 and abs(p[4] + 0.5) < 0.05
    assert 2 * p[1] * p[2] > p[3] ** 2
    assert np.isfinite(res["condition_number"]) and res["condition_number"] < 1e9  # calibration.rs:946-955


def test_jacobi_eigen(oracle):  # calibration.rs:778-867
    a, b, d = 4.0, 1.5, 2.0
    ev, _ = oracle.jacobi_eigen(np.array([[a, b], [b, d]]))
    hd = (a - d) / 2
    disc = math.sqrt(hd * hd + b * b)
    assert np.allclose(sorted(ev), sorted([(a + d) / 2 - disc, (a + d) / 2 + disc]), atol=1e-10)
    A = np.array([[6.0, -1.5, 0.8, 2.1, -0.3], [-1.5, 4.2, 1.1, -0.6, 0.9], [0.8, 1.1, 5.5, 0.4, -1.2],
                  [2.1, -0.6, 0.4, 3.8, 0.7], [-0.3, 0.9, -1.2, 0.7, 2.9]])
    ev, vec = oracle.jacobi_eigen(A)
    assert np.allclose(vec @ vec.T, np.eye(5), atol=1e-8)
    for i in range(5):
        assert np.allclose(A @ vec[i], ev[i] * vec[i], atol=1e-6)
    ev, _ = oracle.jacobi_eigen(np.array([[4.0, 1.0, 5.0], [1.0, 3.0, 4.0], [5.0, 4.0, 9.0]]))
    assert min(abs(ev)) < 1e-6


def test_lm_step_solves_damped_system(oracle):  # calibration.rs:673-703
    rng = np.random.default_rng(0)
    J = rng.normal(size=(30, 5))
    jtj = J.T @ J
    g = rng.normal(size=5)
    dp = oracle.lm_step(jtj, g, 1e-3)
    A = jtj + np.diag(np.diag(jtj)) * 1e-3
    assert np.allclose(A @ dp, -g, atol=1e-9)


def test_bisection_counts_bounded(oracle):
    v, nb = oracle.bates_price(100.0, 330.0, 1 / 365, 0.03, 0.0, [0.01, 0.2, 0.01, 1.0, -0.95, 1.5, -0.3, 0.05],
                               0, 1e-10, stats=True)
    assert np.all(nb <= 199) and np.all(nb >= 0)
