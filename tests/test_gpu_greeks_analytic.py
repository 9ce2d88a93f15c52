"""GPU: all eight Greeks as exact derivatives (ope_batch_greeks_ad with
OPE_FLAG_ANALYTIC_GREEKS) -- the S / r / T sensitivities that ad.rs:751-763
leaves to finite differences, plus gamma, vanna and volga, from one pricing
and one backward pass.

Checked against central differences of the device pricer itself at
tolerance 1e-12 (fourth order, at two step sizes: the analytic value must lie
within three times their disagreement plus the differences' rounding noise),
against differences of the analytic first derivatives (gamma = d delta/dS,
vanna = d vega/dS, volga = d vega/dsqrt(v0)), and against the reference's
own finite-difference Greeks (greeks.rs:19-72, the oracle) within the
truncation error of its 1 % / 0.01 / 1bp / 1-day bumps."""
import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu

S = 100.0
TOL = 1e-12
EPS = 2e-11 * S  # price noise at tol 1e-12 (quadrature decisions), for the differences' noise bars
HP = [0.04, 2.0, 0.04, 0.3, -0.7]
BP = HP + [0.5, -0.1, 0.15]


def _contracts():
    rows = []
    for t in (0.05, 0.25, 1.0, 2.5):
        for k in (75.0, 95.0, 100.0, 110.0, 140.0):
            for ot, q in ((0, 0.0), (1, 0.02)):
                rows.append((S, k, t, 0.03, q, 0.2, ot, 0))
    return np.array(rows, dtype=W.CONTRACT_DTYPE)


def _price(ope, model, con, params):
    """Prices of contracts with one parameter row each."""
    off = np.arange(con.size + 1, dtype=np.int64)
    return ope.price_surfaces(model, con, off, np.atleast_2d(params), tol=TOL)


def _fd4(f, h):
    return (-f(2 * h) + 8 * f(h) - 8 * f(-h) + f(-2 * h)) / (12 * h)


def _fd4_2(f, h):  # second derivative, fourth order
    return (-f(2 * h) + 16 * f(h) - 30 * f(0.0) + 16 * f(-h) - f(-2 * h)) / (12 * h * h)


@pytest.mark.parametrize("bates", [False, True])
def test_analytic_greeks_match_differences_of_the_pricer(ope, bates):
    model = ope.MODEL_BATES if bates else ope.MODEL_HESTON
    p = np.array(BP if bates else HP)
    con = _contracts()
    n = con.size
    g = ope.batch_greeks_ad(model, con, p, tol=TOL, analytic=True)
    P = np.tile(p, (n, 1))
    sig = np.sqrt(p[0])

    def bump(field=None, vol=False):
        """Prices with `field` (or sqrt(v0)) moved by h (an array: one step per contract)."""
        def f(h):
            c, q = con.copy(), P.copy()
            if field is not None:
                c[field] = c[field] + h
            if vol:
                q[:, 0] = (sig + h) ** 2
            return _price(ope, model, c, q)
        return f

    # name: (bumped prices, step per contract, sign of the Greek vs the derivative)
    checks = {
        "delta": (bump("spot"), 0.01 * S * np.sqrt(p[0] * con["expiry"]), 1.0),
        "rho": (bump("rate"), np.full(n, 1e-3), 1.0),
        "theta": (bump("expiry"), 1e-3 * con["expiry"], -1.0),
        "vega": (bump(vol=True), np.full(n, 2e-3 * sig), 1.0),
    }
    worst = {}
    for name, (f, h, sign) in checks.items():
        d1, d2 = sign * _fd4(f, h), sign * _fd4(f, h / 2)
        bar = 3 * np.abs(d1 - d2) + 3 * EPS / (h / 2) + 1e-9 * np.abs(d2)
        err = np.abs(g[name] - d2)
        worst[name] = float(np.max(err / bar))
        assert np.all(err <= bar), (name, float(np.max(err)), worst[name])
    hs = checks["delta"][1]
    g1, g2 = _fd4_2(bump("spot"), hs), _fd4_2(bump("spot"), hs / 2)
    bar = 3 * np.abs(g1 - g2) + 20 * EPS / (hs / 2) ** 2 + 1e-9 * np.abs(g2)
    err = np.abs(g["gamma"] - g2)
    worst["gamma"] = float(np.max(err / bar))
    assert np.all(err <= bar), ("gamma", float(np.max(err)), worst["gamma"])
    print(f"bates={bates}: worst error / bar {worst}")


@pytest.mark.parametrize("bates", [False, True])
def test_second_order_greeks_match_differences_of_first_order(ope, bates):
    """gamma = d delta/dS, vanna = d vega/dS, volga = d vega/dsqrt(v0), the
    first derivatives themselves analytic (their differences carry no price
    noise amplification beyond one order)."""
    model = ope.MODEL_BATES if bates else ope.MODEL_HESTON
    p = np.array(BP if bates else HP)
    con = _contracts()
    g = ope.batch_greeks_ad(model, con, p, tol=TOL, analytic=True)
    hs = 0.01 * S * np.sqrt(p[0] * con["expiry"])
    sig = np.sqrt(p[0])

    def at(ds=0.0, dsig=0.0):
        c = con.copy()
        c["spot"] = c["spot"] + ds * hs
        q = p.copy()
        q[0] = (sig + dsig) ** 2
        return ope.batch_greeks_ad(model, c, q, tol=TOL, analytic=True)

    up, dn = at(ds=1.0), at(ds=-1.0)
    gamma_fd = (up["delta"] - dn["delta"]) / (2 * hs)
    vanna_fd = (up["vega"] - dn["vega"]) / (2 * hs)
    k = 1e-3 * sig
    vu, vd = at(dsig=k), at(dsig=-k)
    volga_fd = (vu["vega"] - vd["vega"]) / (2 * k)
    for name, fd, h in (("gamma", gamma_fd, hs), ("vanna", vanna_fd, hs), ("volga", volga_fd, k)):
        bar = 2e-3 * np.abs(fd) + 1e-6 * np.max(np.abs(fd)) + 1e-9 / h
        err = np.abs(g[name] - fd)
        assert np.all(err <= bar), (name, float(np.max(err / bar)))


@pytest.mark.parametrize("bates", [False, True])
def test_analytic_greeks_agree_with_the_reference_bump_greeks(ope, oracle, bates):
    """In the reference's conventions: greeks.rs:19-72's finite differences
    (the oracle) equal the analytic Greeks up to their own leading truncation
    terms, which the analytic Greeks at the bumped points estimate:
    delta ~ ds^2/6 P_SSS, gamma ~ ds^2/12 P_SSSS, vega ~ dv^2/6 P_vvv (v the
    volatility sqrt(v0)), theta (one-sided, one day) ~ dt/2 P_TT, vanna (a
    cross bump) ~ dv^2/6 P_Svvv + ds^2/6 P_SSSv, volga (a double bump of
    step 2 dv) ~ dv^2/3 P_vvvv; rho's 1bp step leaves 1e-7 relative.
    Expiries from 0.25 years."""
    model = ope.MODEL_BATES if bates else ope.MODEL_HESTON
    p = np.array(BP if bates else HP)
    con = _contracts()
    con = con[con["expiry"] >= 0.25]
    tol = 1e-10
    g = ope.batch_greeks_ad(model, con, p, tol=tol, analytic=True)
    ref = oracle.batch_greeks(con, p, bates, tol=tol)
    ds, dv, dt = 0.01 * S, 0.01, 1.0 / 365.0
    sig = np.sqrt(p[0])

    def at(dS=0.0, dsig=0.0, dT=0.0):
        c = con.copy()
        c["spot"] += dS
        c["expiry"] += dT
        q = p.copy()
        q[0] = (sig + dsig) ** 2
        return ope.batch_greeks_ad(model, c, q, tol=tol, analytic=True)

    su, sd, vu, vd, td = at(dS=ds), at(dS=-ds), at(dsig=dv), at(dsig=-dv), at(dT=-dt)
    trunc = {
        "price": np.zeros(con.size),
        "delta": ds * ds / 6 * np.abs((su["gamma"] - sd["gamma"]) / (2 * ds)),
        "gamma": ds * ds / 12 * np.abs((su["gamma"] - 2 * g["gamma"] + sd["gamma"]) / (ds * ds)),
        "vega": dv * dv / 6 * np.abs((vu["volga"] - vd["volga"]) / (2 * dv)),
        "theta": np.abs(td["theta"] - g["theta"]) / 2,
        "rho": 1e-7 * np.abs(g["rho"]),
        # cross bump: dv^2/6 d3(delta)/dv3 + ds^2/6 d3(vega)/dS3, both from second differences of vanna
        "vanna": np.abs(vu["vanna"] - 2 * g["vanna"] + vd["vanna"]) / 6
                 + np.abs(su["vanna"] - 2 * g["vanna"] + sd["vanna"]) / 6,
        # second difference with step 2 dv: (2 dv)^2/12 P_vvvv, from the second difference of volga
        "volga": np.abs(vu["volga"] - 2 * g["volga"] + vd["volga"]) / 3,
    }
    noise = {"price": 1e-9 * S, "delta": 1e-8, "gamma": 1e-7, "vega": 1e-7, "theta": 1e-6, "rho": 1e-6,
             "vanna": 1e-5, "volga": 1e-4}
    worst = {}
    for i, nm in enumerate(["price", "delta", "gamma", "vega", "theta", "rho", "vanna", "volga"]):
        bar = 2 * trunc[nm] + 1e-6 * np.abs(ref[:, i]) + noise[nm]
        err = np.abs(g[nm] - ref[:, i])
        worst[nm] = float(np.max(err / bar))
        assert np.all(err <= bar), (nm, worst[nm], float(np.max(err)))
    print(f"bates={bates}: worst error / bar vs the reference's bump Greeks {worst}")


def test_analytic_price_and_vega_equal_the_adjoint_path(ope, oracle):
    """The analytic mode's price is the pricing kernel's, and its vega the
    exact dP/dv0 of the parameter adjoint (the AD mode's vega)."""
    con = _contracts()
    a = ope.batch_greeks_ad(ope.MODEL_HESTON, con, HP, tol=1e-10, analytic=True)
    b = ope.batch_greeks_ad(ope.MODEL_HESTON, con, HP, tol=1e-10)
    assert np.array_equal(a["price"], b["price"])
    assert np.allclose(a["vega"], b["vega"], rtol=1e-7, atol=1e-9 * S)
