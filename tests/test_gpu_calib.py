"""GPU: the device Levenberg-Marquardt calibration (calibration.rs:433-569)
and its adjoint Jacobian, against the oracle (the reference's LM with its
finite-difference Jacobian, and forward-mode AD) and against the reference's
own calibration tests (calibration.rs:1020-1071)."""
import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu


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


def _c4_small(oracle, n_surf=6, seed=4):
    def price_fn(con, params, sidx):
        return oracle.batch_price(con, params, False, 1e-8, surf_idx=sidx)
    return W.c4(price_fn, oracle.batch_implied_vol, n_surf=n_surf, seed=seed)


def test_jacobian_matches_forward_ad_and_fd(ope, oracle):
    con, iv, off, true_p, p0 = _c4_small(oracle, n_surf=3)
    J, res = ope.calib_jacobian(ope.MODEL_HESTON, con, iv, off, p0)
    sidx = np.repeat(np.arange(off.size - 1), np.diff(off)).astype(np.int32)
    # forward-mode AD (ad.rs:695-731) / BSM vega at the model IV
    price, grad = oracle.batch_price_gradient(con, p0, False, 1e-8, surf_idx=sidx)
    ivm, ok = oracle.batch_implied_vol(con, price)
    vega = np.array([oracle.bsm_price_and_greeks(oracle.contracts(c["spot"], c["strike"], c["expiry"], c["rate"],
                                                                  c["div_yield"], c["opt_type"], vol=v))[3]
                     for c, v in zip(con, ivm)])
    J_ad = np.where(ok[:, None], grad / vega[:, None], 0.0)
    err = np.abs(J - J_ad)
    assert np.all(err <= 1e-7 * np.abs(J_ad) + 1e-9), float((err / (1e-7 * np.abs(J_ad) + 1e-9)).max())
    # the reference's own Jacobian (central FD on IV residuals, calibration.rs:613-652) per surface
    for s in range(off.size - 1):
        a, b = off[s], off[s + 1]
        J_fd = oracle.jacobian(5, con[a:b], iv[a:b], p0[s])
        rel = np.abs(J[a:b] - J_fd) / np.maximum(np.abs(J_fd), 1e-6)
        assert np.median(rel) < 1e-3 and np.mean(rel < 0.02) > 0.97, (s, float(np.median(rel)))
    # residuals at p0 equal the oracle's IV residuals
    assert np.max(np.abs(res - np.where(ok, ivm - iv, 0.0))) < 1e-9


def test_recovers_params_from_synthetic_surface(ope, oracle):  # calibration.rs:1020-1038, 1040-1050
    true_p = [0.04, 2.0, 0.04, 0.3, -0.5]
    con, iv = _make_quotes(oracle, true_p)
    r = ope.calibrate_heston(con, iv, [0.05, 1.5, 0.05, 0.4, -0.3])
    assert r["converged"] and r["rmse"] < 0.005
    p = r["params"][:5]
    assert abs(p[0] - 0.04) < 0.005 and abs(p[4] + 0.5) < 0.05
    assert 2 * p[1] * p[2] > p[3] ** 2
    assert np.isfinite(r["condition_number"]) and r["condition_number"] < 1e9


def test_recovers_bates_params(ope, oracle):  # calibration.rs:1052-1071
    true_p = [0.04, 2.0, 0.04, 0.3, -0.5, 0.5, -0.1, 0.15]
    con, iv = _make_quotes(oracle, true_p, bates=True)
    r = ope.calibrate_bates(con, iv, [0.05, 1.5, 0.05, 0.4, -0.3, 0.3, -0.05, 0.1])
    assert r["converged"] and r["rmse"] < 0.01
    p = r["params"]
    assert abs(p[0] - 0.04) < 0.01 and 2 * p[1] * p[2] > p[3] ** 2


def test_device_lm_matches_oracle_lm(ope, oracle):
    """Same problems, the oracle running the reference's LM (FD Jacobian)."""
    con, iv, off, true_p, p0 = _c4_small(oracle, n_surf=4, seed=9)
    got = ope.calibrate_surfaces(ope.MODEL_HESTON, con, iv, off, p0)
    ref = oracle.calibrate_many(5, con, iv, off, p0)
    for s in range(off.size - 1):
        g, r = got[s], ref[s]
        # both stop at the optimum: by the gradient/step tests, or -- at the noise floor of the
        # objective, where no step lowers the SSE any more -- on the damping cap (calibration.rs:537)
        assert g["status"] in (1, 2), (s, g["status"])
        # same optimum: fit quality to 1e-7 vol points, well-identified params closely
        assert abs(g["rmse"] - r["rmse"]) < 1e-7, (s, g["rmse"], r["rmse"])
        assert abs(g["params"][0] - r["params"][0]) < 1e-4 and abs(g["params"][4] - r["params"][4]) < 1e-3


def test_graph_rerun_is_deterministic(ope, oracle):
    con, iv, off, true_p, p0 = _c4_small(oracle, n_surf=5, seed=21)
    a = ope.calibrate_surfaces(ope.MODEL_HESTON, con, iv, off, p0)
    b = ope.calibrate_surfaces(ope.MODEL_HESTON, con, iv, off, p0)
    assert a.tobytes() == b.tobytes()
    # a surface alone gives the same fit as inside the batch
    s = 2
    alone = ope.calibrate_surfaces(ope.MODEL_HESTON, con[off[s]:off[s + 1]], iv[off[s]:off[s + 1]],
                                   [0, off[s + 1] - off[s]], p0[s:s + 1])
    assert alone[0].tobytes() == a[s].tobytes()


def test_bates_jacobian_jump_columns_match_pure_fd(ope, oracle):  # calibration.rs:1133-1171
    """The device Jacobian's lambda / mu_j / sigma_j columns against central
    differences (h = 1e-4) of the IV residual computed independently, with the
    device pricer and the device IV solver, at the reference's 2 % bar."""
    p = np.array([0.045, 1.8, 0.045, 0.35, -0.55, 0.4, -0.08, 0.12])
    con, iv = _make_quotes(oracle, p, bates=True)
    J, _ = ope.calib_jacobian(ope.MODEL_BATES, con, iv, [0, iv.size], p[None, :])

    def resid(q):
        px = ope.batch_bates(con, q)
        ivm, ok = ope.batch_implied_vol(con, px)
        return np.where(ok, ivm - iv, 0.0)

    h = 1e-4
    for col in (5, 6, 7):
        up, dn = p.copy(), p.copy()
        up[col] += h
        dn[col] -= h
        fd = (resid(up) - resid(dn)) / (2.0 * h)
        err = np.abs(J[:, col] - fd) / np.maximum(np.abs(fd), 1e-6)
        assert np.all(err < 0.02), (col, float(err.max()))
