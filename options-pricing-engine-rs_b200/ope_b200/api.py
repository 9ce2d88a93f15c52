"""Host-side mirror of the reference crate's pricing API over the C ABI.

Names, argument order and meaning follow the reference's public surface
(lib.rs:18-35): ``heston_price`` / ``bates_price`` (heston.rs:61, bates.rs:29),
``batch_heston`` / ``batch_bates`` / ``batch_heston_greeks`` /
``batch_bates_greeks`` (batch.rs:23-48) and the records ``OptionType``,
``OptionContract``, ``PricingResult``, ``HestonParams``, ``BatesParams``
(types.rs).  Where the reference panics this raises ``OpeError``; there is no
CPU fallback.  The quadrature tolerance defaults to the reference's 1e-8
(heston.rs:228); every entry point also takes ``tol=``.

Beyond the reference: ``price_surfaces`` (many surfaces, one persistent
launch) and ``*_device`` variants that take torch CUDA tensors already
resident in HBM and run stream-ordered on the current torch stream.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import MODEL_BATES, MODEL_HESTON, OpeError, Options, check, load
from .workloads import CONTRACT_DTYPE

REF_TOL = 1e-8

RESULT_DTYPE = np.dtype([(k, "<f8") for k in ("price", "delta", "gamma", "vega", "theta", "rho", "vanna", "volga")])


class OptionType(enum.IntEnum):  # types.rs:5-13
    Call = 0
    Put = 1

    def sign(self) -> float:
        return 1.0 if self == OptionType.Call else -1.0


@dataclass
class OptionContract:  # types.rs:16-25
    spot: float
    strike: float
    expiry: float
    rate: float
    div_yield: float
    vol: float
    opt_type: OptionType = OptionType.Call


@dataclass
class HestonParams:  # types.rs:48-63
    v0: float
    kappa: float
    theta: float
    sigma: float
    rho: float

    def feller_ok(self) -> bool:
        return 2.0 * self.kappa * self.theta > self.sigma * self.sigma

    def as_array(self) -> np.ndarray:
        return np.array([self.v0, self.kappa, self.theta, self.sigma, self.rho], dtype=np.float64)


@dataclass
class BatesParams:  # types.rs:66-72
    heston: HestonParams
    lambda_: float
    mu_j: float
    sigma_j: float

    def as_array(self) -> np.ndarray:
        return np.concatenate([self.heston.as_array(), [self.lambda_, self.mu_j, self.sigma_j]]).astype(np.float64)


@dataclass
class PricingResult:  # types.rs:29-39
    price: float = 0.0
    delta: float = 0.0
    gamma: float = 0.0
    vega: float = 0.0
    theta: float = 0.0
    rho: float = 0.0
    vanna: float = 0.0
    volga: float = 0.0


def _params_array(params, model: int) -> np.ndarray:
    if isinstance(params, (HestonParams, BatesParams)):
        arr = params.as_array()
    else:
        arr = np.ascontiguousarray(params, dtype=np.float64)
    want = 8 if model == MODEL_BATES else 5
    if arr.shape[-1] != want:
        raise ValueError(f"expected {want} parameters per set, got shape {arr.shape}")
    return np.ascontiguousarray(arr, dtype=np.float64)


def contracts_array(contracts) -> np.ndarray:
    """OptionContract list / structured array -> contiguous ope_contract records."""
    if isinstance(contracts, np.ndarray) and contracts.dtype == CONTRACT_DTYPE:
        return np.ascontiguousarray(contracts)
    out = np.zeros(len(contracts), CONTRACT_DTYPE)
    for i, c in enumerate(contracts):
        out[i] = (c.spot, c.strike, c.expiry, c.rate, c.div_yield, c.vol, int(c.opt_type), 0)
    return out


def _opts(tol: float, flags: int = 0, stream: int = 0) -> Options:
    return Options(tol=float(tol), flags=flags, reserved=0, stream=stream or None)


def heston_price(spot, strike, expiry, rate, div_yield, params, opt_type=OptionType.Call, tol=REF_TOL) -> float:
    """heston.rs:61-72."""
    return float(batch_heston([OptionContract(spot, strike, expiry, rate, div_yield, 0.0, OptionType(opt_type))],
                              params, tol=tol)[0])


def bates_price(spot, strike, expiry, rate, div_yield, params, opt_type=OptionType.Call, tol=REF_TOL) -> float:
    """bates.rs:29-39."""
    return float(batch_bates([OptionContract(spot, strike, expiry, rate, div_yield, 0.0, OptionType(opt_type))],
                             params, tol=tol)[0])


def _batch(model: int, contracts, params, tol: float) -> np.ndarray:
    con = contracts_array(contracts)
    p = _params_array(params, model)
    out = np.empty(con.size, dtype=np.float64)
    if con.size == 0:
        return out
    o = _opts(tol)
    check(load().ope_batch_price_ex(model, con.ctypes.data, con.size, p.ctypes.data, out.ctypes.data,
                                    ctypes.byref(o)))
    return out


def batch_heston(contracts, params, tol=REF_TOL) -> np.ndarray:
    """batch.rs:23-27 — one parameter set, prices in input order."""
    return _batch(MODEL_HESTON, contracts, params, tol)


def batch_bates(contracts, params, tol=REF_TOL) -> np.ndarray:
    """batch.rs:38-42."""
    return _batch(MODEL_BATES, contracts, params, tol)


def _batch_greeks(model: int, contracts, params, tol: float) -> np.ndarray:
    con = contracts_array(contracts)
    p = _params_array(params, model)
    out = np.zeros(con.size, dtype=RESULT_DTYPE)
    if con.size == 0:
        return out
    if tol == REF_TOL:
        fn = load().ope_batch_bates_greeks if model == MODEL_BATES else load().ope_batch_heston_greeks
        check(fn(con.ctypes.data, con.size, p.ctypes.data, out.ctypes.data))
    else:
        o = _opts(tol)
        check(load().ope_batch_greeks_ex(model, con.ctypes.data, con.size, p.ctypes.data, out.ctypes.data,
                                         ctypes.byref(o)))
    return out


def batch_heston_greeks(contracts, params, tol=REF_TOL) -> np.ndarray:
    """batch.rs:32-36 (bump-and-reprice, greeks.rs:19-72).  Structured array of PricingResult."""
    return _batch_greeks(MODEL_HESTON, contracts, params, tol)


def batch_bates_greeks(contracts, params, tol=REF_TOL) -> np.ndarray:
    """batch.rs:44-48."""
    return _batch_greeks(MODEL_BATES, contracts, params, tol)


def batch_greeks_ad(model: int, contracts, params, tol=REF_TOL, analytic: bool = False) -> np.ndarray:
    """ad.rs:736-795 / 809-865 for many contracts under one parameter set: vega and
    volga from the exact d price / d v0 (adjoint kernel), the rest by the
    reference's finite differences.  analytic=True: all eight Greeks as exact
    derivatives (OPE_FLAG_ANALYTIC_GREEKS) from one pricing and one backward
    pass.  Structured array of PricingResult."""
    con = contracts_array(contracts)
    p = _params_array(params, model)
    out = np.zeros(con.size, dtype=RESULT_DTYPE)
    if con.size == 0:
        return out
    o = _opts(tol, _lib.FLAG_ANALYTIC_GREEKS if analytic else 0)
    check(load().ope_batch_greeks_ad(model, con.ctypes.data, con.size, p.ctypes.data, out.ctypes.data,
                                     ctypes.byref(o)))
    return out


def heston_greeks_ad(spot, strike, expiry, rate, div_yield, params, opt_type=OptionType.Call, tol=REF_TOL):
    """ad.rs:736-795 (one contract): a PricingResult record."""
    c = [OptionContract(spot, strike, expiry, rate, div_yield, 0.0, OptionType(opt_type))]
    return batch_greeks_ad(MODEL_HESTON, c, params, tol)[0]


def bates_greeks_ad(spot, strike, expiry, rate, div_yield, heston, lam, mu_j, sigma_j, opt_type=OptionType.Call,
                    tol=REF_TOL):
    """ad.rs:809-865 (one contract, the reference's argument order): a PricingResult record."""
    c = [OptionContract(spot, strike, expiry, rate, div_yield, 0.0, OptionType(opt_type))]
    hp = _params_array(heston, MODEL_HESTON)
    return batch_greeks_ad(MODEL_BATES, c, np.concatenate([hp, [lam, mu_j, sigma_j]]), tol)[0]


def heston_greeks_ad5(spot, strike, expiry, rate, div_yield, params, opt_type=OptionType.Call, tol=REF_TOL):
    """ad.rs heston_greeks_ad5: the reference's joint five-parameter pass returns the
    same PricingResult as heston_greeks_ad (ad.rs:1295-1322 checks exactly that),
    so it maps to the same device computation."""
    return heston_greeks_ad(spot, strike, expiry, rate, div_yield, params, opt_type, tol)


def bates_jump_sensitivities_ad(spot, strike, expiry, rate, div_yield, heston, lam, mu_j, sigma_j,
                                opt_type=OptionType.Call, tol=REF_TOL):
    """ad.rs:882-895 (one contract): (price, d_lambda, d_mu_j, d_sigma_j) from the
    reverse-mode adjoint."""
    c = [OptionContract(spot, strike, expiry, rate, div_yield, 0.0, OptionType(opt_type))]
    hp = _params_array(heston, MODEL_HESTON)
    p = np.concatenate([hp, [lam, mu_j, sigma_j]])[None, :]
    price, grad = price_gradient_surfaces(MODEL_BATES, c, [0, 1], p, tol)
    return float(price[0]), float(grad[0, 5]), float(grad[0, 6]), float(grad[0, 7])


def price_surfaces(model: int, contracts, surf_offsets, params, tol=REF_TOL, out=None,
                   bisections=None) -> np.ndarray:
    """Many surfaces (one parameter set each) in ONE persistent launch.

    ``out`` (float64, n) may be a caller-owned (e.g. pinned) buffer; with
    ``bisections`` (int32, 2n) the per-integral bisection counts are returned too.
    """
    con = contracts_array(contracts)
    off = np.ascontiguousarray(surf_offsets, dtype=np.int64)
    p = _params_array(params, model)
    n_surf = off.size - 1
    if p.ndim != 2 or p.shape[0] != n_surf:
        raise ValueError("params must be (n_surf, 5|8)")
    if out is None:
        out = np.empty(con.size, dtype=np.float64)
    if con.size == 0:
        return out
    o = _opts(tol)
    if bisections is None:
        check(load().ope_price_surfaces(model, con.ctypes.data, con.size, off.ctypes.data, n_surf, p.ctypes.data,
                                        out.ctypes.data, ctypes.byref(o)))
    else:
        assert bisections.dtype == np.int32 and bisections.size == 2 * con.size
        check(load().ope_price_surfaces_stats(model, con.ctypes.data, con.size, off.ctypes.data, n_surf,
                                              p.ctypes.data, out.ctypes.data, bisections.ctypes.data,
                                              ctypes.byref(o)))
    return out


def price_gradient_surfaces(model: int, contracts, surf_offsets, params, tol=REF_TOL):
    """Prices and d price / d params (n x 5 Heston, n x 8 Bates) by the adjoint kernel.

    The parameter order is (v0, kappa, theta, sigma, rho[, lambda, mu_j, sigma_j]);
    the same derivatives ad.rs:695-731 / 882-895 compute by forward-mode AD.
    """
    con = contracts_array(contracts)
    off = np.ascontiguousarray(surf_offsets, dtype=np.int64)
    p = _params_array(params, model)
    n_surf = off.size - 1
    if p.ndim != 2 or p.shape[0] != n_surf:
        raise ValueError("params must be (n_surf, 5|8)")
    dim = p.shape[1]
    price = np.empty(con.size, dtype=np.float64)
    grad = np.empty((con.size, dim), dtype=np.float64)
    if con.size == 0:
        return price, grad
    o = _opts(tol)
    check(load().ope_price_gradient_surfaces(model, con.ctypes.data, con.size, off.ctypes.data, n_surf,
                                             p.ctypes.data, price.ctypes.data, grad.ctypes.data, ctypes.byref(o)))
    return price, grad


CALIB_RESULT_DTYPE = np.dtype([
    ("params", "<f8", (8,)), ("rmse", "<f8"), ("max_err", "<f8"), ("condition_number", "<f8"),
    ("weakest_direction", "<f8", (8,)), ("iters", "<i4"), ("converged", "<i4"), ("early_stopped", "<i4"),
    ("status", "<i4"),
])  # include/ope.h ope_calib_result = calibration.rs:44-68 CalibResult


def calibrate_surfaces(model: int, quotes, iv_market, surf_offsets, p0, weights=None, tol=REF_TOL) -> np.ndarray:
    """Levenberg-Marquardt in IV space for many quote surfaces at once (calibration.rs:433-569).

    Returns one CALIB_RESULT_DTYPE record per surface; ``params[:dim]`` are the fitted
    (v0, kappa, theta, sigma, rho[, lambda, mu_j, sigma_j]).
    """
    con = contracts_array(quotes)
    iv = np.ascontiguousarray(iv_market, dtype=np.float64)
    off = np.ascontiguousarray(surf_offsets, dtype=np.int64)
    p = _params_array(p0, model)
    n_surf = off.size - 1
    if p.ndim != 2 or p.shape[0] != n_surf:
        raise ValueError("p0 must be (n_surf, 5|8)")
    if iv.size != con.size:
        raise ValueError("iv_market must have one entry per quote")
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    out = np.zeros(n_surf, dtype=CALIB_RESULT_DTYPE)
    o = _opts(tol)
    check(load().ope_calibrate_surfaces(model, con.ctypes.data, iv.ctypes.data, None if w is None else w.ctypes.data,
                                        con.size, off.ctypes.data, n_surf, p.ctypes.data, out.ctypes.data,
                                        ctypes.byref(o)))
    return out


def calibrate_heston(quotes, iv_market, p0, weights=None, tol=REF_TOL):
    """calibration.rs:204-206 (one surface)."""
    return calibrate_surfaces(MODEL_HESTON, quotes, iv_market, [0, len(iv_market)], np.atleast_2d(
        _params_array(p0, MODEL_HESTON)), weights, tol)[0]


def calibrate_bates(quotes, iv_market, p0, weights=None, tol=REF_TOL):
    """calibration.rs:208-210 (one surface)."""
    return calibrate_surfaces(MODEL_BATES, quotes, iv_market, [0, len(iv_market)], np.atleast_2d(
        _params_array(p0, MODEL_BATES)), weights, tol)[0]


MULTISTART_RESULT_DTYPE = np.dtype([
    ("best", CALIB_RESULT_DTYPE), ("n_restarts", "<i4"), ("n_converged", "<i4"), ("n_pruned", "<i4"),
    ("best_restart", "<i4"),
])  # include/ope.h ope_multistart_result = calibration.rs:70-76 MultistartResult

GLOBAL_RESULT_DTYPE = np.dtype([
    ("best", CALIB_RESULT_DTYPE), ("de_best_sse", "<f8"), ("de_generations", "<i4"), ("n_pop", "<i4"),
])  # include/ope.h ope_global_result = calibration.rs:296-300 GlobalCalibResult


def _calib_inputs(model, quotes, iv_market, surf_offsets, weights):
    con = contracts_array(quotes)
    iv = np.ascontiguousarray(iv_market, dtype=np.float64)
    off = np.ascontiguousarray(surf_offsets, dtype=np.int64)
    if iv.size != con.size:
        raise ValueError("iv_market must have one entry per quote")
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    return con, iv, off, w


def _per_surface(x, n_surf, model, name):
    p = _params_array(x, model)
    if p.ndim == 1:
        p = np.ascontiguousarray(np.broadcast_to(p, (n_surf, p.size)))
    if p.shape[0] != n_surf:
        raise ValueError(f"{name} must be (n_surf, 5|8)")
    return p


def calibrate_surfaces_reg(model: int, quotes, iv_market, surf_offsets, p0, prior, reg_weight, weights=None,
                           tol=REF_TOL) -> np.ndarray:
    """LM with a Tikhonov pull toward `prior` (calibration.rs:220-230), many surfaces at once."""
    con, iv, off, w = _calib_inputs(model, quotes, iv_market, surf_offsets, weights)
    n_surf = off.size - 1
    p = _per_surface(p0, n_surf, model, "p0")
    pr = _per_surface(prior, n_surf, model, "prior")
    rw = np.ascontiguousarray(np.broadcast_to(np.asarray(reg_weight, np.float64), (n_surf,)))
    out = np.zeros(n_surf, dtype=CALIB_RESULT_DTYPE)
    o = _opts(tol)
    check(load().ope_calibrate_surfaces_reg(model, con.ctypes.data, iv.ctypes.data,
                                            None if w is None else w.ctypes.data, con.size, off.ctypes.data, n_surf,
                                            p.ctypes.data, pr.ctypes.data, rw.ctypes.data, out.ctypes.data,
                                            ctypes.byref(o)))
    return out


def calibrate_multistart(model: int, quotes, iv_market, surf_offsets, p0, n_restarts: int, seed: int, weights=None,
                         shared_best0=None, return_restarts: bool = False, tol=REF_TOL):
    """calibration.rs:246-314 for many surfaces at once.  Returns MULTISTART_RESULT_DTYPE
    records (and, with return_restarts, every restart's CALIB_RESULT_DTYPE record,
    shape (n_surf, max(n_restarts, 1)))."""
    con, iv, off, w = _calib_inputs(model, quotes, iv_market, surf_offsets, weights)
    n_surf = off.size - 1
    p = _per_surface(p0, n_surf, model, "p0")
    nr = max(int(n_restarts), 1)
    out = np.zeros(n_surf, dtype=MULTISTART_RESULT_DTYPE)
    allr = np.zeros((n_surf, nr), dtype=CALIB_RESULT_DTYPE) if return_restarts else None
    sb = None if shared_best0 is None else np.ascontiguousarray(
        np.broadcast_to(np.asarray(shared_best0, np.float64), (n_surf,)))
    o = _opts(tol)
    check(load().ope_calibrate_multistart(model, con.ctypes.data, iv.ctypes.data,
                                          None if w is None else w.ctypes.data, con.size, off.ctypes.data, n_surf,
                                          p.ctypes.data, int(n_restarts), ctypes.c_uint64(int(seed) & (2**64 - 1)),
                                          None if sb is None else sb.ctypes.data, out.ctypes.data,
                                          None if allr is None else allr.ctypes.data, ctypes.byref(o)))
    return (out, allr) if return_restarts else out


def calibrate_global(model: int, quotes, iv_market, surf_offsets, n_pop: int, n_gen: int, seed: int, weights=None,
                     prior=None, reg_weight=None, tol=REF_TOL) -> np.ndarray:
    """calibration.rs:316-427 (differential evolution + LM polish, regularised when
    `prior` is given) for many surfaces at once; GLOBAL_RESULT_DTYPE records."""
    con, iv, off, w = _calib_inputs(model, quotes, iv_market, surf_offsets, weights)
    n_surf = off.size - 1
    pr = rw = None
    if prior is not None:
        pr = _per_surface(prior, n_surf, model, "prior")
        rw = np.ascontiguousarray(np.broadcast_to(np.asarray(reg_weight, np.float64), (n_surf,)))
    out = np.zeros(n_surf, dtype=GLOBAL_RESULT_DTYPE)
    o = _opts(tol)
    check(load().ope_calibrate_global(model, con.ctypes.data, iv.ctypes.data, None if w is None else w.ctypes.data,
                                      con.size, off.ctypes.data, n_surf, int(n_pop), int(n_gen),
                                      ctypes.c_uint64(int(seed) & (2**64 - 1)),
                                      None if pr is None else pr.ctypes.data, None if rw is None else rw.ctypes.data,
                                      out.ctypes.data, ctypes.byref(o)))
    return out


def _one(model, quotes):
    return [0, len(quotes)]


def calibrate_heston_regularized(quotes, iv_market, p0, prior, reg_weight, weights=None, tol=REF_TOL):
    """calibration.rs:220-224 (one surface)."""
    return calibrate_surfaces_reg(MODEL_HESTON, quotes, iv_market, _one(0, iv_market), p0, prior, reg_weight,
                                  weights, tol)[0]


def calibrate_bates_regularized(quotes, iv_market, p0, prior, reg_weight, weights=None, tol=REF_TOL):
    """calibration.rs:226-230 (one surface)."""
    return calibrate_surfaces_reg(MODEL_BATES, quotes, iv_market, _one(1, iv_market), p0, prior, reg_weight,
                                  weights, tol)[0]


def calibrate_heston_multistart(quotes, iv_market, p0, n_restarts, seed, weights=None, tol=REF_TOL):
    """calibration.rs:246-250 (one surface)."""
    return calibrate_multistart(MODEL_HESTON, quotes, iv_market, _one(0, iv_market), p0, n_restarts, seed,
                                weights, tol=tol)[0]


def calibrate_bates_multistart(quotes, iv_market, p0, n_restarts, seed, weights=None, tol=REF_TOL):
    """calibration.rs:252-256 (one surface)."""
    return calibrate_multistart(MODEL_BATES, quotes, iv_market, _one(1, iv_market), p0, n_restarts, seed,
                                weights, tol=tol)[0]


def calibrate_heston_global(quotes, iv_market, n_pop, n_gen, seed, weights=None, tol=REF_TOL):
    """calibration.rs:316-320 (one surface)."""
    return calibrate_global(MODEL_HESTON, quotes, iv_market, _one(0, iv_market), n_pop, n_gen, seed, weights,
                            tol=tol)[0]


def calibrate_bates_global(quotes, iv_market, n_pop, n_gen, seed, weights=None, tol=REF_TOL):
    """calibration.rs:322-326 (one surface)."""
    return calibrate_global(MODEL_BATES, quotes, iv_market, _one(1, iv_market), n_pop, n_gen, seed, weights,
                            tol=tol)[0]


def calibrate_heston_global_regularized(quotes, iv_market, n_pop, n_gen, seed, prior, reg_weight, weights=None,
                                        tol=REF_TOL):
    """calibration.rs:335-340 (one surface)."""
    return calibrate_global(MODEL_HESTON, quotes, iv_market, _one(0, iv_market), n_pop, n_gen, seed, weights,
                            prior, reg_weight, tol)[0]


def calibrate_bates_global_regularized(quotes, iv_market, n_pop, n_gen, seed, prior, reg_weight, weights=None,
                                       tol=REF_TOL):
    """calibration.rs:342-347 (one surface)."""
    return calibrate_global(MODEL_BATES, quotes, iv_market, _one(1, iv_market), n_pop, n_gen, seed, weights,
                            prior, reg_weight, tol)[0]


def calib_jacobian(model: int, quotes, iv_market, surf_offsets, params, tol=REF_TOL):
    """The device IV-space Jacobian (n x dim) and IV residuals at params (calibration.rs:613-652)."""
    con = contracts_array(quotes)
    iv = np.ascontiguousarray(iv_market, dtype=np.float64)
    off = np.ascontiguousarray(surf_offsets, dtype=np.int64)
    p = _params_array(params, model)
    dim = p.shape[-1]
    jac = np.zeros((con.size, dim))
    res = np.zeros(con.size)
    o = _opts(tol)
    check(load().ope_calib_jacobian(model, con.ctypes.data, iv.ctypes.data, con.size, off.ctypes.data, off.size - 1,
                                    p.ctypes.data, jac.ctypes.data, res.ctypes.data, ctypes.byref(o)))
    return jac, res


def batch_implied_vol(contracts, market_prices):
    """batch.rs:51-56 on the device: (iv, ok); ok[i] is False where the reference returns None."""
    con = contracts_array(contracts)
    px = np.ascontiguousarray(market_prices, dtype=np.float64)
    iv = np.zeros(con.size)
    ok = np.zeros(con.size, np.int32)
    if con.size:
        check(load().ope_batch_implied_vol(con.ctypes.data, con.size, px.ctypes.data, iv.ctypes.data, ok.ctypes.data,
                                           None))
    return iv, ok.astype(bool)


def measure_fp64_peak() -> tuple[float, float]:
    """(flop/s, ms) of the DFMA throughput probe on the current device."""
    f, ms = ctypes.c_double(), ctypes.c_double()
    check(load().ope_measure_fp64_peak(ctypes.byref(f), ctypes.byref(ms)))
    return f.value, ms.value


def _tune_rows(entries) -> list[dict]:
    return [{"max_contracts": int(e.max_contracts) if e.max_contracts < 2 ** 63 else None,
             "warps_per_block": int(e.shape.warps_per_block), "deepest_first": bool(e.shape.deepest_first),
             "occupancy": float(e.shape.occupancy), "per_unit": int(e.shape.per_unit),
             "ms_default": float(e.ms_default), "ms_tuned": float(e.ms_tuned)}
            for e in entries]


def autotune(model: int, quick: bool = False) -> list[dict]:
    """Measure the pricing kernel's launch shapes on this device (ope_autotune)
    and install the per-size-class table; returns its rows (the last class,
    max_contracts None, is every larger call)."""
    entries = (_lib.TuneEntry * _lib.TUNE_CLASSES)()
    check(load().ope_autotune(model, _lib.TUNE_QUICK if quick else 0, entries))
    return _tune_rows(entries)


def set_autotune(enabled: bool) -> None:
    """Use the tuned tables (True) or the default launch shape (False)."""
    check(load().ope_set_autotune(1 if enabled else 0))


def set_tune_table(model: int, rows: list[dict]) -> None:
    """Install a table (rows as autotune / tune_table return them) on this device."""
    if len(rows) != _lib.TUNE_CLASSES:
        raise ValueError(f"expected {_lib.TUNE_CLASSES} rows")
    entries = (_lib.TuneEntry * _lib.TUNE_CLASSES)()
    for e, r in zip(entries, rows):
        e.shape.warps_per_block = int(r["warps_per_block"])
        e.shape.deepest_first = int(bool(r["deepest_first"]))
        e.shape.occupancy = float(r["occupancy"])
        e.shape.per_unit = int(r.get("per_unit", 0))
        e.ms_default = float(r.get("ms_default", 0.0))
        e.ms_tuned = float(r.get("ms_tuned", 0.0))
    check(load().ope_set_tune_table(model, entries))


def last_per_unit() -> int:
    """Contracts per unit of this thread's last plain pricing launch (1: one
    per unit; automatic launches report the run probe's choice)."""
    v = ctypes.c_int32()
    check(load().ope_last_per_unit(ctypes.byref(v)))
    return int(v.value)


def tune_table(model: int) -> tuple[list[dict], bool]:
    """The current device's table for `model`, and whether it was tuned."""
    entries = (_lib.TuneEntry * _lib.TUNE_CLASSES)()
    tuned = ctypes.c_int32()
    check(load().ope_get_tune_table(model, entries, ctypes.byref(tuned)))
    return _tune_rows(entries), bool(tuned.value)


TRACE_FIELDS = 39  # OPE_TRACE_FIELDS
MAX_STEPS = 200    # OPE_MAX_PANELS: the first panel + at most 199 bisections


def trace_integral(model: int, contract, params, which: int, tol=REF_TOL):
    """Step-by-step record of the device's greedy GK15 quadrature
    (heston.rs:193-212) on integral `which` (0 = P1, 1 = P2) of one contract:
    a (steps, TRACE_FIELDS) array -- per step a, b, ew of the bisected panel,
    kl, el, kr, er of its children, the running error and total, then the 15
    left and 15 right integrand values -- and the integral."""
    if isinstance(contract, np.void):
        contract = np.array([contract], dtype=CONTRACT_DTYPE)
    elif not isinstance(contract, np.ndarray):
        contract = [contract]
    con = contracts_array(contract)
    if con.size != 1:
        raise ValueError("trace_integral takes one contract")
    par = _params_array(params, model)
    out = np.zeros((MAX_STEPS, TRACE_FIELDS))
    n, integral = ctypes.c_int32(), ctypes.c_double()
    check(load().ope_trace_integral(model, con.ctypes.data, par.ctypes.data, int(which), float(tol), out.ctypes.data,
                                    MAX_STEPS, ctypes.byref(n), ctypes.byref(integral)))
    return out[:n.value], integral.value


# ---------------------------------------------------------------- device path
def _torch_stream_ptr() -> int:
    import torch

    return torch.cuda.current_stream().cuda_stream


def price_surfaces_device(model: int, d_contracts, n: int, d_offsets, n_surf: int, d_params, d_out,
                          tol=REF_TOL, stream: int | None = None) -> None:
    """Stream-ordered persistent launch over device buffers (torch tensors or raw pointers)."""
    ptr = lambda t: t if isinstance(t, int) else t.data_ptr()  # noqa: E731
    o = _opts(tol, _lib.FLAG_DEVICE_PTRS, _torch_stream_ptr() if stream is None else stream)
    check(load().ope_price_surfaces(model, ptr(d_contracts), n, ptr(d_offsets), n_surf, ptr(d_params), ptr(d_out),
                                    ctypes.byref(o)))


def price_gradient_surfaces_device(model: int, d_contracts, n: int, d_offsets, n_surf: int, d_params, d_prices,
                                   d_grad, tol=REF_TOL, stream: int | None = None) -> None:
    """Stream-ordered adjoint launch (prices + n x dim gradient) over device buffers."""
    ptr = lambda t: t if isinstance(t, int) else t.data_ptr()  # noqa: E731
    o = _opts(tol, _lib.FLAG_DEVICE_PTRS, _torch_stream_ptr() if stream is None else stream)
    check(load().ope_price_gradient_surfaces(model, ptr(d_contracts), n, ptr(d_offsets), n_surf, ptr(d_params),
                                             ptr(d_prices), ptr(d_grad), ctypes.byref(o)))


def batch_price_device(model: int, d_contracts, n: int, d_params, d_out, tol=REF_TOL,
                       stream: int | None = None) -> None:
    """Stream-ordered plain (single parameter set) launch over device buffers."""
    ptr = lambda t: t if isinstance(t, int) else t.data_ptr()  # noqa: E731
    o = _opts(tol, _lib.FLAG_DEVICE_PTRS, _torch_stream_ptr() if stream is None else stream)
    check(load().ope_batch_price_ex(model, ptr(d_contracts), n, ptr(d_params), ptr(d_out), ctypes.byref(o)))


def set_workspace_limit(nbytes: int) -> None:
    """Cap the device workspace of the calling thread's calls (0: no cap); a call
    needing more raises OpeError(OPE_ERR_OUT_OF_MEMORY) before allocating."""
    check(load().ope_set_workspace_limit(int(nbytes)))


def workspace_bytes() -> int:
    """Device workspace bytes the calling thread holds."""
    return int(load().ope_workspace_bytes())


def kernel_launch_count() -> int:
    return int(load().ope_kernel_launch_count())


def device_info() -> tuple[int, int, int]:
    sm, ma, mi = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(load().ope_device_info(ctypes.byref(sm), ctypes.byref(ma), ctypes.byref(mi)))
    return sm.value, ma.value, mi.value


__all__ = [
    "OptionType", "OptionContract", "HestonParams", "BatesParams", "PricingResult", "OpeError",
    "heston_price", "bates_price", "batch_heston", "batch_bates", "batch_heston_greeks", "batch_bates_greeks",
    "price_surfaces", "price_surfaces_device", "batch_price_device", "contracts_array", "REF_TOL",
    "MODEL_HESTON", "MODEL_BATES", "RESULT_DTYPE", "kernel_launch_count", "device_info", "measure_fp64_peak", "price_gradient_surfaces",
    "price_gradient_surfaces_device", "batch_greeks_ad", "heston_greeks_ad", "bates_greeks_ad",
    "heston_greeks_ad5", "bates_jump_sensitivities_ad", "set_workspace_limit", "workspace_bytes",
    "CALIB_RESULT_DTYPE", "batch_implied_vol", "calibrate_surfaces", "calibrate_heston", "calibrate_bates", "calib_jacobian",
    "MULTISTART_RESULT_DTYPE", "GLOBAL_RESULT_DTYPE", "calibrate_surfaces_reg", "calibrate_multistart",
    "calibrate_global", "calibrate_heston_regularized", "calibrate_bates_regularized", "calibrate_heston_multistart",
    "calibrate_bates_multistart", "calibrate_heston_global", "calibrate_bates_global",
    "calibrate_heston_global_regularized", "calibrate_bates_global_regularized", "trace_integral",
    "autotune", "set_autotune", "tune_table", "set_tune_table", "last_per_unit",
]
