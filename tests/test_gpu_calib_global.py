"""GPU: Tikhonov-regularised, multistart and differential-evolution
calibration on the device (calibration.rs:204-427) against the oracle and
against the reference's own calibration tests (calibration.rs:870-1234).

The device LM differentiates exactly (adjoint / BSM vega); the reference
differentiates the Heston columns by central differences.  The oracle runs
both: jac_mode=1 restates the device's Jacobian, so the device is compared
with it restart for restart (same pruning, same winner, same iteration
counts up to the pricing's rounding); jac_mode=0 is the reference's own LM,
against which the device must reach the same fits."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRUE_H = [0.04, 2.0, 0.04, 0.3, -0.5]
TRUE_B = TRUE_H + [0.5, -0.1, 0.15]
P0_H = [0.05, 1.5, 0.05, 0.4, -0.3]
PRIOR_B = [0.035, 1.8, 0.04, 0.35, -0.45, 0.4, -0.08, 0.12]


def _make_quotes(oracle, p, bates=False):  # calibration.rs:980-1018
    rows, ivs = [], []
    for t in (0.25, 0.5, 1.0):
        for k in (80.0, 90.0, 95.0, 100.0, 105.0, 110.0, 120.0):
            ot = 0 if k >= 100.0 else 1
            px = (oracle.bates_price if bates else oracle.heston_price)(100.0, k, t, 0.03, 0.0, p, ot)
            c = oracle.contracts(100.0, k, t, 0.03, 0.0, ot, vol=0.2)
            iv = oracle.implied_vol(c, px)
            if iv is not None and 0.01 < iv < 2.0:
                rows.append(c[0])
                ivs.append(iv)
    return np.array(rows), np.array(ivs)


@pytest.fixture(scope="module")
def hq(oracle):
    return _make_quotes(oracle, TRUE_H)


@pytest.fixture(scope="module")
def bq(oracle):
    return _make_quotes(oracle, TRUE_B, bates=True)


def _close(a, b, rtol, atol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return bool(np.all(np.abs(a - b) <= atol + rtol * np.abs(b)))


# ---- Tikhonov ---------------------------------------------------------------
def test_regularized_matches_oracle(ope, oracle, hq):
    con, iv = hq
    prior = [0.045, 1.8, 0.045, 0.32, -0.45]
    g = ope.calibrate_heston_regularized(con, iv, P0_H, prior, 1e-3)
    o1 = oracle.calibrate_ex(5, con, iv, P0_H, prior=prior, reg_weight=1e-3, jac_mode=1)
    o0 = oracle.calibrate(5, con, iv, P0_H, prior=prior, reg_weight=1e-3)
    assert g["converged"] == o1["converged"] and g["iters"] == o1["iters"]
    assert _close(g["params"][:5], o1["params"][:5], 1e-7, 1e-10)
    assert abs(g["rmse"] - o1["rmse"]) < 1e-10 and abs(g["rmse"] - o0["rmse"]) < 1e-7
    assert _close(g["params"][:5], o0["params"][:5], 1e-4, 1e-7)
    # diagnostics stay data-only (calibration.rs:541-568)
    assert abs(g["condition_number"] / o1["condition_number"] - 1.0) < 1e-6


def test_regularization_does_not_hurt_a_well_identified_case(ope, hq):  # calibration.rs:911-935
    con, iv = hq
    unreg = ope.calibrate_heston(con, iv, P0_H)
    reg = ope.calibrate_heston_regularized(con, iv, P0_H, [0.045, 1.8, 0.045, 0.32, -0.45], 1e-3)
    assert reg["rmse"] < 0.002 and abs(reg["params"][0] - unreg["params"][0]) < 0.005


def test_regularized_batch_equals_single_surface_calls(ope, hq):
    con, iv = hq
    n = iv.size
    priors = np.array([[0.045, 1.8, 0.045, 0.32, -0.45], [0.03, 2.5, 0.05, 0.25, -0.6], TRUE_H])
    w = np.array([1e-3, 1e-2, 0.0])
    res = ope.calibrate_surfaces_reg(ope.MODEL_HESTON, np.concatenate([con] * 3), np.concatenate([iv] * 3),
                                     [0, n, 2 * n, 3 * n], np.array([P0_H] * 3), priors, w)
    for s in range(3):
        one = ope.calibrate_heston_regularized(con, iv, P0_H, priors[s], w[s])
        assert res[s].tobytes() == one.tobytes()
    plain = ope.calibrate_heston(con, iv, P0_H)  # weight 0: the Tikhonov rows add exact zeros
    assert np.array_equal(res[2]["params"], plain["params"]) and res[2]["iters"] == plain["iters"]


# ---- multistart --------------------------------------------------------------
def test_multistart_matches_oracle_restart_for_restart(ope, oracle, hq):
    con, iv = hq
    bad = [0.25, 6.0, 0.3, 0.15, 0.6]
    out, allr = ope.calibrate_multistart(ope.MODEL_HESTON, con, iv, [0, iv.size], bad, 8, 12345,
                                         return_restarts=True)
    best, oall, n_conv, n_pruned, bi = oracle.calibrate_multistart(5, con, iv, bad, 8, 12345, jac_mode=1)
    m = out[0]
    assert (m["n_restarts"], m["n_converged"], m["n_pruned"], m["best_restart"]) == (8, n_conv, n_pruned, bi)
    assert list(allr[0]["iters"]) == list(oall["iters"])
    assert list(allr[0]["early_stopped"]) == list(oall["early_stopped"])
    assert list(allr[0]["converged"]) == list(oall["converged"])
    assert abs(m["best"]["rmse"] - best["rmse"]) < 1e-9
    assert _close(m["best"]["params"][:5], best["params"][:5], 1e-6, 1e-9)
    # the reference's LM reaches the same winner
    best0, _, n_conv0, _, bi0 = oracle.calibrate_multistart(5, con, iv, bad, 8, 12345, jac_mode=0)
    assert bi0 == bi and abs(best0["rmse"] - best["rmse"]) < 1e-8


def test_multistart_beats_bad_single_start(ope, hq):  # calibration.rs:1216-1234
    con, iv = hq
    bad = [0.25, 6.0, 0.3, 0.15, 0.6]
    single = ope.calibrate_heston(con, iv, bad)
    multi = ope.calibrate_heston_multistart(con, iv, bad, 8, 12345)
    assert multi["n_converged"] >= 1
    assert multi["best"]["rmse"] <= single["rmse"] + 1e-9
    assert multi["best"]["rmse"] < 0.01


def test_prune_mechanism(ope, hq):  # calibration.rs:1176-1214
    con, iv = hq
    off = [0, iv.size]
    hopeless = ope.calibrate_multistart(ope.MODEL_HESTON, con, iv, off, [0.3, 7.5, 0.35, 0.12, 0.8], 1, 0,
                                        shared_best0=1e-10)[0]
    assert hopeless["n_pruned"] == 1 and hopeless["best"]["early_stopped"] == 1
    assert hopeless["best"]["iters"] < 200 and hopeless["best"]["converged"] == 0
    assert hopeless["best"]["status"] == 4
    ok = ope.calibrate_multistart(ope.MODEL_HESTON, con, iv, off, P0_H, 1, 0, shared_best0=float("inf"))[0]
    assert ok["n_pruned"] == 0 and ok["best"]["converged"] == 1 and ok["best"]["rmse"] < 0.005


def test_multistart_surfaces_are_independent(ope, hq, bq):
    con, iv = hq
    n = iv.size
    iv2 = iv + 0.01 * np.sin(np.arange(n))
    both = ope.calibrate_multistart(ope.MODEL_HESTON, np.concatenate([con, con]), np.concatenate([iv, iv2]),
                                    [0, n, 2 * n], np.array([[0.25, 6.0, 0.3, 0.15, 0.6], P0_H]), 4, 99)
    one = ope.calibrate_multistart(ope.MODEL_HESTON, con, iv2, [0, n], P0_H, 4, 99)
    assert both[1].tobytes() == one[0].tobytes()


# ---- differential evolution ------------------------------------------------------
def test_de_matches_oracle(ope, oracle, hq):
    con, iv = hq
    g = ope.calibrate_heston_global(con, iv, 40, 60, 777)
    o, de_sse, pop, fit = oracle.calibrate_global(5, con, iv, 40, 60, 777, jac_mode=1)
    assert g["n_pop"] == 40 and g["de_generations"] == 60
    assert abs(g["de_best_sse"] - de_sse) <= 1e-9 * de_sse + 1e-15
    assert _close(g["best"]["params"][:5], o["params"][:5], 1e-6, 1e-9)
    assert abs(g["best"]["rmse"] - o["rmse"]) < 1e-9


def test_de_global_recovers_heston_params(ope, hq):  # calibration.rs:1073-1099
    con, iv = hq
    g = ope.calibrate_heston_global(con, iv, 40, 60, 777)
    p = g["best"]["params"]
    assert g["best"]["rmse"] < 0.01 and abs(p[0] - 0.04) < 0.01 and abs(p[4] + 0.5) < 0.1
    assert 2.0 * p[1] * p[2] > p[3] * p[3]
    assert g["best"]["rmse"] <= math.sqrt(g["de_best_sse"] / iv.size) + 1e-9


def test_de_global_bates_lands_where_the_reference_recorded(ope, oracle, bq):  # calibration.rs:1101-1131, 937-976
    con, iv = bq
    g = ope.calibrate_bates_global(con, iv, 60, 80, 999)
    p = g["best"]["params"]
    assert g["best"]["rmse"] < 0.005 and 2.0 * p[1] * p[2] > p[3] * p[3]
    assert round(p[0], 2) == 1.64 and round(p[1]) == 21  # "v0=1.64 vs true 0.04, kappa=21 vs true 2"
    cn = g["best"]["condition_number"]
    assert cn > 1e10 or not math.isfinite(cn)
    o, de_sse, _, _ = oracle.calibrate_global(8, con, iv, 60, 80, 999, jac_mode=1)
    assert abs(g["de_best_sse"] - de_sse) <= 1e-9 * de_sse + 1e-15


def test_regularization_recovers_plausible_params(ope, bq):  # calibration.rs:870-909
    con, iv = bq
    g = ope.calibrate_bates_global_regularized(con, iv, 60, 80, 999, PRIOR_B, 1e-3)
    p = g["best"]["params"]
    assert g["best"]["rmse"] < 0.005 and g["best"]["condition_number"] < 1e9
    assert abs(p[0] - 0.04) < 0.01 and abs(p[1] - 2.0) < 0.5 and abs(p[5] - 0.5) < 0.15
    assert abs(p[6] + 0.1) < 0.05 and abs(p[7] - 0.15) < 0.05


def test_de_surfaces_are_independent_and_zero_generations(ope, oracle, hq):
    con, iv = hq
    n = iv.size
    iv2 = iv + 0.005
    both = ope.calibrate_global(ope.MODEL_HESTON, np.concatenate([con, con]), np.concatenate([iv, iv2]),
                                [0, n, 2 * n], 24, 5, 3)
    one = ope.calibrate_global(ope.MODEL_HESTON, con, iv2, [0, n], 24, 5, 3)
    assert both[1].tobytes() == one[0].tobytes()
    z = ope.calibrate_heston_global(con, iv, 10, 0, 5)  # population floored at 4 x dim; no generations
    o, de_sse, _, _ = oracle.calibrate_global(5, con, iv, 10, 0, 5, jac_mode=1)
    assert z["n_pop"] == 20 and z["de_generations"] == 0
    assert abs(z["de_best_sse"] - de_sse) <= 1e-9 * de_sse + 1e-15
