"""TEST INFRASTRUCTURE ONLY — ctypes binding of the CPU oracle (ope_oracle.cpp).

The oracle restates the reference crate's Heston/Bates pricing path on the
CPU (heston.rs, bates.rs, batch.rs, greeks.rs, iv.rs, bsm.rs, math.rs, the
forward-mode AD of ad.rs and the LM engine of calibration.rs).  It is the
checker for the CUDA product path and the timed CPU baseline; the product
library never imports it.

Parity status: the reference is Rust and no Rust toolchain exists in this
environment, so the oracle cannot be diffed against the reference binary.  It
is pinned instead by (1) every invariant the reference's own tests assert on
this path (put-call parity, static no-arbitrage grids, the zero vol-of-vol
BSM limit, Bates -> Heston as jumps vanish, AD price == pricer price, batch ==
scalar, fast_csqrt == principal sqrt), re-run against the oracle in
tests/test_oracle.py, and (2) independent high-precision known answers
(mpmath Gil-Pelaez integrals, tests/golden/).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libope_oracle.so")

CONTRACT_DTYPE = np.dtype(
    [
        ("spot", "<f8"),
        ("strike", "<f8"),
        ("expiry", "<f8"),
        ("rate", "<f8"),
        ("div_yield", "<f8"),
        ("vol", "<f8"),
        ("opt_type", "<i4"),
        ("pad", "<i4"),
    ],
    align=False,
)
assert CONTRACT_DTYPE.itemsize == 56

CALIB_OUT_DTYPE = np.dtype(
    [
        ("params", "<f8", (8,)),
        ("rmse", "<f8"),
        ("max_err", "<f8"),
        ("condition_number", "<f8"),
        ("weakest", "<f8", (8,)),
        ("iters", "<i4"),
        ("converged", "<i4"),
        ("early_stopped", "<i4"),
        ("pad", "<i4"),
    ]
)

REF_TOL = 1e-8  # heston.rs:228 — the reference's hard-coded quadrature tolerance

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off, OpenMP)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
        os.path.join(_HERE, "ope_oracle.cpp")
    ):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        vp = ctypes.c_void_p
        d, i, i64 = ctypes.c_double, ctypes.c_int, ctypes.c_int64
        u64, u64p = ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)
        sig = {
            "orc_fast_csqrt": (None, [d, d, dp]),
            "orc_stable_cf": (None, [d, d, d, d, dp, dp]),
            "orc_jump_cf": (None, [d, d, d, dp, dp]),
            "orc_cf_integrand": (d, [d, d, d, d, d, dp, i]),
            "orc_heston_price": (d, [d, d, d, d, d, dp, i, d, ip]),
            "orc_bates_price": (d, [d, d, d, d, d, dp, i, d, ip]),
            "orc_batch_price": (None, [vp, i64, ip, dp, i, d, dp, ip, i]),
            "orc_trace_integral": (i, [vp, dp, i, i, d, dp, i, dp]),
            "orc_batch_greeks": (None, [vp, i64, dp, i, d, dp, i]),
            "orc_npdf": (d, [d]),
            "orc_ncdf": (d, [d]),
            "orc_ncdf_inv": (d, [d]),
            "orc_bsm_price": (d, [vp]),
            "orc_bsm_price_and_greeks": (None, [vp, dp]),
            "orc_implied_vol": (i, [vp, d, dp]),
            "orc_batch_implied_vol": (None, [vp, i64, dp, dp, ip, i]),
            "orc_forward_pass": (None, [d, d, d, d, d, dp, i, i, i, d, d, d, i, d, dp, dp]),
            "orc_price_gradient": (None, [vp, dp, i, d, dp, dp]),
            "orc_batch_price_gradient": (None, [vp, i64, ip, dp, i, d, dp, dp, i]),
            "orc_greeks_ad": (None, [vp, dp, i, d, dp]),
            "orc_calibrate": (None, [i, vp, dp, dp, i, dp, dp, d, vp]),
            "orc_calibrate_many": (None, [i, vp, dp, ctypes.POINTER(ctypes.c_int64), i, dp, vp, i]),
            "orc_jacobian": (None, [i, vp, dp, i, dp, dp]),
            "orc_jacobi_eigen": (None, [dp, i, dp, dp]),
            "orc_lm_step": (None, [dp, dp, d, i, dp]),
            "orc_calibrate_ex": (None, [i, vp, dp, dp, i, dp, dp, d, i, d, vp]),
            "orc_calibrate_multistart": (None, [i, vp, dp, dp, i, dp, i, u64, i, d, vp, vp, ip, i]),
            "orc_calibrate_global": (None, [i, vp, dp, dp, i, i, i, u64, dp, d, i, vp, dp, dp, dp, ip, i]),
            "orc_splitmix64": (u64, [u64]),
            "orc_small_rng_u64": (None, [u64, i, u64p]),
            "orc_xoshiro_from_state": (None, [u64p, i, u64p]),
            "orc_rng_gen_range_f64": (None, [u64, d, d, i, dp]),
            "orc_rng_gen_range_usize": (None, [u64, u64, u64, i, u64p]),
            "orc_random_guess": (None, [i, u64, dp]),
            "orc_calib_out_size": (i, []),
            "orc_max_threads": (i, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        assert L.orc_calib_out_size() == CALIB_OUT_DTYPE.itemsize
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def heston_vec(p) -> np.ndarray:
    if isinstance(p, dict):
        p = [p["v0"], p["kappa"], p["theta"], p["sigma"], p["rho"]]
    return np.ascontiguousarray(p, dtype=np.float64)


def contracts(spot, strike, expiry, rate, div_yield, opt_type, vol=0.2) -> np.ndarray:
    """Build a contract array (numpy broadcasting over the fields)."""
    b = np.broadcast_arrays(
        np.asarray(spot, float), np.asarray(strike, float), np.asarray(expiry, float),
        np.asarray(rate, float), np.asarray(div_yield, float), np.asarray(vol, float),
        np.asarray(opt_type, np.int32),
    )
    out = np.zeros(b[0].size, dtype=CONTRACT_DTYPE)
    for name, arr in zip(["spot", "strike", "expiry", "rate", "div_yield", "vol", "opt_type"], b):
        out[name] = arr.ravel()
    return out


def fast_csqrt(z: complex) -> complex:
    out = np.zeros(2)
    lib().orc_fast_csqrt(z.real, z.imag, _dptr(out))
    return complex(out[0], out[1])


def stable_cf(phi: complex, t: float, r: float, hp) -> complex:
    out = np.zeros(2)
    h = heston_vec(hp)
    lib().orc_stable_cf(phi.real, phi.imag, t, r, _dptr(h), _dptr(out))
    return complex(out[0], out[1])


def jump_cf(phi: complex, t: float, bp) -> complex:
    out = np.zeros(2)
    b = np.ascontiguousarray(bp, dtype=np.float64)
    lib().orc_jump_cf(phi.real, phi.imag, t, _dptr(b), _dptr(out))
    return complex(out[0], out[1])


def heston_price(spot, strike, expiry, rate, div_yield, hp, opt_type=0, tol=REF_TOL, stats=False):
    h = heston_vec(hp)
    nb = np.zeros(2, np.int32)
    v = lib().orc_heston_price(spot, strike, expiry, rate, div_yield, _dptr(h), int(opt_type), tol, _iptr(nb))
    return (v, nb) if stats else v


def bates_price(spot, strike, expiry, rate, div_yield, bp, opt_type=0, tol=REF_TOL, stats=False):
    b = np.ascontiguousarray(bp, dtype=np.float64)
    nb = np.zeros(2, np.int32)
    v = lib().orc_bates_price(spot, strike, expiry, rate, div_yield, _dptr(b), int(opt_type), tol, _iptr(nb))
    return (v, nb) if stats else v


def batch_price(con: np.ndarray, params: np.ndarray, bates: bool, tol: float = REF_TOL,
                surf_idx: np.ndarray | None = None, nthreads: int = 0, stats: bool = False):
    """Price many contracts; params is (n_surf, 5|8); surf_idx maps contract -> row."""
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    params = np.ascontiguousarray(params, dtype=np.float64)
    n = con.size
    out = np.empty(n)
    nb = np.zeros(2 * n, np.int32) if stats else None
    si = None if surf_idx is None else np.ascontiguousarray(surf_idx, dtype=np.int32)
    lib().orc_batch_price(con.ctypes.data, n, _iptr(si), _dptr(params), int(bates), tol, _dptr(out),
                          _iptr(nb), int(nthreads))
    return (out, nb) if stats else out


TRACE_FIELDS = 39  # per step: a, b, ew, kl, el, kr, er, err, total, 15 left + 15 right integrand values
MAX_STEPS = 200     # the first panel + at most 199 bisections (heston.rs:194)


def trace_integral(c, params, bates: bool, which: int, tol: float = REF_TOL):
    """Step-by-step record of adaptive_gk (heston.rs:193-212) on integral
    `which` (0 = P1, 1 = P2) of contract `c`: a (steps, TRACE_FIELDS) array
    and the integral.  Same fields as the device library's trace."""
    c = np.ascontiguousarray(np.atleast_1d(c), dtype=CONTRACT_DTYPE)
    params = np.ascontiguousarray(params, dtype=np.float64)
    out = np.zeros((MAX_STEPS, TRACE_FIELDS))
    integral = np.zeros(1)
    n = lib().orc_trace_integral(c.ctypes.data, _dptr(params), int(bates), int(which), tol, _dptr(out), MAX_STEPS,
                                 _dptr(integral))
    return out[:n], float(integral[0])


def batch_greeks(con: np.ndarray, params, bates: bool, tol: float = REF_TOL, nthreads: int = 0) -> np.ndarray:
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    p = np.ascontiguousarray(params, dtype=np.float64)
    out = np.empty((con.size, 8))
    lib().orc_batch_greeks(con.ctypes.data, con.size, _dptr(p), int(bates), tol, _dptr(out), int(nthreads))
    return out


def ncdf(x):
    return lib().orc_ncdf(float(x))


def npdf(x):
    return lib().orc_npdf(float(x))


def ncdf_inv(p):
    return lib().orc_ncdf_inv(float(p))


def bsm_price(c) -> float:
    c = np.ascontiguousarray(c, dtype=CONTRACT_DTYPE).reshape(1)
    return lib().orc_bsm_price(c.ctypes.data)


def bsm_price_and_greeks(c) -> np.ndarray:
    c = np.ascontiguousarray(c, dtype=CONTRACT_DTYPE).reshape(1)
    out = np.zeros(8)
    lib().orc_bsm_price_and_greeks(c.ctypes.data, _dptr(out))
    return out


def implied_vol(c, market_price: float):
    c = np.ascontiguousarray(c, dtype=CONTRACT_DTYPE).reshape(1)
    out = np.zeros(1)
    ok = lib().orc_implied_vol(c.ctypes.data, float(market_price), _dptr(out))
    return float(out[0]) if ok else None


def batch_implied_vol(con, prices, nthreads: int = 0):
    """iv.rs:14-20 over many contracts: (iv, ok) arrays."""
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    px = np.ascontiguousarray(prices, dtype=np.float64)
    out = np.zeros(con.size)
    ok = np.zeros(con.size, np.int32)
    lib().orc_batch_implied_vol(con.ctypes.data, con.size, _dptr(px), _dptr(out), _iptr(ok), int(nthreads))
    return out, ok.astype(bool)


def forward_pass(s, k, t, r, q, hp, opt_type, active, jump=None, jump_active=-1, tol=REF_TOL):
    """ad.rs:695-731.  jump None = Off; (l, m, s) = Const; with jump_active>=0 = Active."""
    h = heston_vec(hp)
    pv, dv = np.zeros(1), np.zeros(1)
    if jump is None:
        mode, jl, jm, js = 0, 0.0, 0.0, 0.0
    else:
        jl, jm, js = jump
        mode = 2 if jump_active >= 0 else 1
    lib().orc_forward_pass(s, k, t, r, q, _dptr(h), int(opt_type), int(active), mode, jl, jm, js,
                           int(jump_active), tol, _dptr(pv), _dptr(dv))
    return float(pv[0]), float(dv[0])


def price_gradient(c, params, bates: bool, tol: float = REF_TOL):
    c = np.ascontiguousarray(c, dtype=CONTRACT_DTYPE).reshape(1)
    p = np.ascontiguousarray(params, dtype=np.float64)
    price = np.zeros(1)
    grad = np.zeros(8 if bates else 5)
    lib().orc_price_gradient(c.ctypes.data, _dptr(p), int(bates), tol, _dptr(price), _dptr(grad))
    return float(price[0]), grad


def batch_price_gradient(con, params, bates: bool, tol: float = REF_TOL, surf_idx=None, nthreads: int = 0):
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    p = np.ascontiguousarray(params, dtype=np.float64)
    n = con.size
    price = np.empty(n)
    grad = np.empty((n, 8 if bates else 5))
    si = None if surf_idx is None else np.ascontiguousarray(surf_idx, dtype=np.int32)
    lib().orc_batch_price_gradient(con.ctypes.data, n, _iptr(si), _dptr(p), int(bates), tol, _dptr(price),
                                   _dptr(grad), int(nthreads))
    return price, grad


def greeks_ad(c, params, bates: bool, tol: float = REF_TOL) -> np.ndarray:
    c = np.ascontiguousarray(c, dtype=CONTRACT_DTYPE).reshape(1)
    p = np.ascontiguousarray(params, dtype=np.float64)
    out = np.zeros(8)
    lib().orc_greeks_ad(c.ctypes.data, _dptr(p), int(bates), tol, _dptr(out))
    return out


def calibrate(dim: int, con, iv_market, p0, weight=None, prior=None, reg_weight=0.0):
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    iv = np.ascontiguousarray(iv_market, dtype=np.float64)
    w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
    p0 = np.ascontiguousarray(p0, dtype=np.float64)
    pr = None if prior is None else np.ascontiguousarray(prior, dtype=np.float64)
    out = np.zeros(1, CALIB_OUT_DTYPE)
    lib().orc_calibrate(dim, con.ctypes.data, _dptr(iv), None if w is None else _dptr(w), con.size, _dptr(p0),
                        None if pr is None else _dptr(pr), float(reg_weight), out.ctypes.data)
    return out[0]


def _quotes(con, iv_market, weight):
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    iv = np.ascontiguousarray(iv_market, dtype=np.float64)
    w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
    return con, iv, w


def calibrate_ex(dim: int, con, iv_market, p0, weight=None, prior=None, reg_weight=0.0, jac_mode: int = 0,
                 shared_best=float("nan")):
    """calibrate_inner with every option: Tikhonov prior, the Jacobian variant
    (0 = the reference's FD/AD, 1 = exact, as the device LM), and a fixed
    shared best SSE to prune against (NaN = no pruning)."""
    con, iv, w = _quotes(con, iv_market, weight)
    p0 = np.ascontiguousarray(p0, dtype=np.float64)
    pr = None if prior is None else np.ascontiguousarray(prior, dtype=np.float64)
    out = np.zeros(1, CALIB_OUT_DTYPE)
    lib().orc_calibrate_ex(dim, con.ctypes.data, _dptr(iv), None if w is None else _dptr(w), con.size, _dptr(p0),
                           None if pr is None else _dptr(pr), float(reg_weight), int(jac_mode), float(shared_best),
                           out.ctypes.data)
    return out[0]


def calibrate_multistart(dim: int, con, iv_market, p0, n_restarts: int, seed: int, weight=None, jac_mode: int = 0,
                         shared_best0=float("inf"), nthreads: int = 0):
    """calibration.rs:266-314 with the restarts in lockstep.  Returns
    (best record, all records, n_converged, n_pruned, best index)."""
    con, iv, w = _quotes(con, iv_market, weight)
    p0 = np.ascontiguousarray(p0, dtype=np.float64)
    nr = max(int(n_restarts), 1)
    best = np.zeros(1, CALIB_OUT_DTYPE)
    allr = np.zeros(nr, CALIB_OUT_DTYPE)
    cnt = np.zeros(3, np.int32)
    lib().orc_calibrate_multistart(dim, con.ctypes.data, _dptr(iv), None if w is None else _dptr(w), con.size,
                                   _dptr(p0), nr, ctypes.c_uint64(int(seed) & (2**64 - 1)), int(jac_mode),
                                   float(shared_best0), best.ctypes.data, allr.ctypes.data, _iptr(cnt), int(nthreads))
    return best[0], allr, int(cnt[0]), int(cnt[1]), int(cnt[2])


def calibrate_global(dim: int, con, iv_market, n_pop: int, n_gen: int, seed: int, weight=None, prior=None,
                     reg_weight=0.0, jac_mode: int = 0, nthreads: int = 0):
    """calibration.rs:349-427.  Returns (polished record, de_best_sse,
    final population, final fitness)."""
    con, iv, w = _quotes(con, iv_market, weight)
    pr = None if prior is None else np.ascontiguousarray(prior, dtype=np.float64)
    np_used = max(int(n_pop), 4 * dim)
    out = np.zeros(1, CALIB_OUT_DTYPE)
    sse = np.zeros(1)
    pop = np.zeros((np_used, dim))
    fit = np.zeros(np_used)
    npu = np.zeros(1, np.int32)
    lib().orc_calibrate_global(dim, con.ctypes.data, _dptr(iv), None if w is None else _dptr(w), con.size,
                               int(n_pop), int(n_gen), ctypes.c_uint64(int(seed) & (2**64 - 1)),
                               None if pr is None else _dptr(pr), float(reg_weight), int(jac_mode), out.ctypes.data,
                               _dptr(sse), _dptr(pop), _dptr(fit), _iptr(npu), int(nthreads))
    assert int(npu[0]) == np_used
    return out[0], float(sse[0]), pop, fit


def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def splitmix64(x: int) -> int:
    return int(lib().orc_splitmix64(ctypes.c_uint64(x & (2**64 - 1))))


def small_rng_u64(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint64)
    lib().orc_small_rng_u64(ctypes.c_uint64(seed & (2**64 - 1)), n, _u64p(out))
    return out


def xoshiro_from_state(state4, n: int) -> np.ndarray:
    st = np.ascontiguousarray(state4, dtype=np.uint64)
    out = np.zeros(n, np.uint64)
    lib().orc_xoshiro_from_state(_u64p(st), n, _u64p(out))
    return out


def rng_gen_range_f64(seed: int, lo: float, hi: float, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().orc_rng_gen_range_f64(ctypes.c_uint64(seed & (2**64 - 1)), lo, hi, n, _dptr(out))
    return out


def rng_gen_range_usize(seed: int, lo: int, hi: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint64)
    lib().orc_rng_gen_range_usize(ctypes.c_uint64(seed & (2**64 - 1)), lo, hi, n, _u64p(out))
    return out


def random_guess(dim: int, seed: int) -> np.ndarray:
    """CalibModel::random_guess from SmallRng::seed_from_u64(seed)."""
    out = np.zeros(dim)
    lib().orc_random_guess(dim, ctypes.c_uint64(seed & (2**64 - 1)), _dptr(out))
    return out


def calibrate_many(dim: int, con, iv_market, offsets, p0s, nthreads: int = 0) -> np.ndarray:
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    iv = np.ascontiguousarray(iv_market, dtype=np.float64)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    p0s = np.ascontiguousarray(p0s, dtype=np.float64)
    n_surf = off.size - 1
    out = np.zeros(n_surf, CALIB_OUT_DTYPE)
    lib().orc_calibrate_many(dim, con.ctypes.data, _dptr(iv), off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                             n_surf, _dptr(p0s), out.ctypes.data, int(nthreads))
    return out


def jacobian(dim: int, con, iv_market, p) -> np.ndarray:
    con = np.ascontiguousarray(con, dtype=CONTRACT_DTYPE)
    iv = np.ascontiguousarray(iv_market, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    j = np.zeros((con.size, dim))
    lib().orc_jacobian(dim, con.ctypes.data, _dptr(iv), con.size, _dptr(p), _dptr(j))
    return j


def jacobi_eigen(a: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    ev = np.zeros(n)
    evec = np.zeros((n, n))
    lib().orc_jacobi_eigen(_dptr(a), n, _dptr(ev), _dptr(evec))
    return ev, evec


def lm_step(jtj, grad, lam):
    jtj = np.ascontiguousarray(jtj, dtype=np.float64)
    grad = np.ascontiguousarray(grad, dtype=np.float64)
    n = grad.size
    dp = np.zeros(n)
    lib().orc_lm_step(_dptr(jtj), _dptr(grad), float(lam), n, _dptr(dp))
    return dp


def max_threads() -> int:
    return lib().orc_max_threads()
