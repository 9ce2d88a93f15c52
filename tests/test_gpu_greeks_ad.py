"""GPU: AD Greeks (ad.rs:736-795 heston_greeks_ad, 809-865 bates_greeks_ad)
on the device against the oracle's restatement of the same formulas, and the
reference's own AD tests (ad.rs:907-965, 1364-1420).

Bars: every Greek within the finite-difference amplification of a 1e-9 S
price tolerance (as for the bump Greeks), plus, for vega and volga, the
adjoint's 1e-7 relative bar on d price / d v0 carried through their
formulas."""
import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu

S = 100.0
PRICE_TOL = 1e-9 * S
P = [0.04, 2.0, 0.04, 0.3, -0.7]          # ad.rs:903-905
JUMPS = [0.5, -0.1, 0.15]                 # ad.rs:927
NAMES = ["price", "delta", "gamma", "vega", "theta", "rho", "vanna", "volga"]
AMP = {"price": 1, "delta": 1, "gamma": 4, "vega": 100, "theta": 2 * 365, "rho": 1e4, "vanna": 200, "volga": 2e4}


def _grid():
    rows = []
    for t in (0.02, 0.1, 0.5, 1.0, 2.0):                  # ad.rs:926-927
        for k in (70.0, 85.0, 100.0, 115.0, 130.0):
            for ot in (0, 1):
                rows.append((S, k, t, 0.05, 0.0, 0.2, ot, 0))
    return np.array(rows, dtype=W.CONTRACT_DTYPE)


@pytest.mark.parametrize("bates", [False, True])
def test_greeks_ad_match_oracle(ope, oracle, bates):
    con = _grid()
    p = P + JUMPS if bates else P
    got = ope.batch_greeks_ad(ope.MODEL_BATES if bates else ope.MODEL_HESTON, con, p)
    ref = np.array([oracle.greeks_ad(c, p, bates) for c in con])
    for i, nm in enumerate(NAMES):
        bar = PRICE_TOL * AMP[nm]
        if nm == "vega":
            bar = bar + 1e-7 * np.abs(ref[:, 3])
        if nm == "volga":
            bar = bar + 1e-7 * 2.0 * (np.abs(ref[:, 3]) + 1.0) / 0.02
        err = np.abs(got[nm] - ref[:, i])
        assert np.all(err <= bar), (nm, float(err.max()))


def test_bates_ad_matches_heston_ad_when_jumps_off(ope):  # ad.rs:907-917
    h = ope.heston_greeks_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 0)
    b = ope.bates_greeks_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 0.0, 0.0, 1e-8, 0)
    assert abs(h["price"] - b["price"]) < 1e-6
    assert abs(h["vega"] - b["vega"]) < 1e-4


def test_ad_price_matches_standard_across_wings(ope):  # ad.rs:919-939, 1388-1406
    con = _grid()
    con = con[con["opt_type"] == 0]
    hb = ope.batch_greeks_ad(ope.MODEL_HESTON, con, P)
    bb = ope.batch_greeks_ad(ope.MODEL_BATES, con, P + JUMPS)
    assert np.max(np.abs(hb["price"] - ope.batch_heston(con, P))) < 1e-6
    assert np.max(np.abs(bb["price"] - ope.batch_bates(con, P + JUMPS))) < 1e-6


def test_price_matches_standard(ope):  # ad.rs:1364-1371
    ad = ope.heston_greeks_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 0)
    c = [ope.OptionContract(100.0, 100.0, 1.0, 0.05, 0.0, 0.0, ope.OptionType.Call)]
    std = ope.batch_heston_greeks(c, P)[0]
    assert abs(ad["price"] - std["price"]) < 1e-10


def test_vega_close_to_bump(ope):  # ad.rs:1410-1419, 941-953
    c = [ope.OptionContract(100.0, 100.0, 1.0, 0.05, 0.0, 0.0, ope.OptionType.Call)]
    for model, p, bump in ((ope.MODEL_HESTON, P, ope.batch_heston_greeks),
                           (ope.MODEL_BATES, P + JUMPS, ope.batch_bates_greeks)):
        ad = ope.batch_greeks_ad(model, c, p)[0]
        std = bump(c, p)[0]
        assert abs(ad["vega"] - std["vega"]) / max(abs(std["vega"]), 1e-10) < 0.01


def test_greeks_signs(ope):  # ad.rs:1373-1386, 955-965
    r = ope.heston_greeks_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 0)
    assert 0.0 < r["delta"] < 1.0 and r["gamma"] > 0.0 and r["vega"] > 0.0 and r["rho"] > 0.0
    r = ope.heston_greeks_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 1)
    assert -1.0 < r["delta"] < 0.0
    r = ope.bates_greeks_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 0.5, -0.1, 0.15, 0)
    assert 0.0 < r["delta"] < 1.0 and r["gamma"] > 0.0 and r["vega"] > 0.0


def test_greeks_ad_empty_and_device_pointers(ope, oracle):
    import torch

    assert ope.batch_greeks_ad(ope.MODEL_HESTON, np.zeros(0, W.CONTRACT_DTYPE), P).size == 0
    con = _grid()
    host = ope.batch_greeks_ad(ope.MODEL_BATES, con, P + JUMPS)
    d_con = torch.from_numpy(con.view(np.uint8).copy()).cuda()
    d_par = torch.tensor(P + JUMPS, dtype=torch.float64, device="cuda")
    d_out = torch.zeros(con.size * 8, dtype=torch.float64, device="cuda")
    import ctypes

    o = ope._lib.Options(tol=ope.REF_TOL, flags=ope._lib.FLAG_DEVICE_PTRS, reserved=0,
                         stream=torch.cuda.current_stream().cuda_stream)
    ope._lib.check(ope._lib.load().ope_batch_greeks_ad(ope.MODEL_BATES, d_con.data_ptr(), con.size,
                                                       d_par.data_ptr(), d_out.data_ptr(), ctypes.byref(o)))
    torch.cuda.synchronize()
    dev = d_out.cpu().numpy().reshape(-1, 8)
    assert np.array_equal(dev, np.stack([host[nm] for nm in NAMES], axis=1))


def test_aliases_of_the_reference_api(ope, oracle):  # ad.rs:1295-1322, 882-895
    a = ope.heston_greeks_ad5(100.0, 100.0, 1.0, 0.05, 0.0, P, 0)
    b = ope.heston_greeks_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 0)
    assert a.tobytes() == b.tobytes()
    price, dl, dm, ds = ope.bates_jump_sensitivities_ad(100.0, 100.0, 1.0, 0.05, 0.0, P, 0.5, -0.1, 0.15, 0)
    c = oracle.contracts(100.0, 100.0, 1.0, 0.05, 0.0, 0)
    rp, rg = oracle.price_gradient(c, P + JUMPS, True)
    assert abs(price - rp) <= PRICE_TOL
    for got, ref in zip((dl, dm, ds), rg[5:8]):
        assert abs(got - ref) <= 1e-7 * abs(ref) + 1e-9 * S
    assert dm < 0.0  # ad.rs:1022-1027
