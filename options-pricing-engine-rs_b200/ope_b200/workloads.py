"""Seeded synthetic workloads for the Heston/Bates CF pricing path.

No public dataset is involved: the reference prices user-supplied contract
chains (batch.rs:23-48), so every workload here is generated from a fixed seed
with the shapes, sizes and value ranges of the five benchmark configurations:

* ``c1``  one Heston surface, 15 strikes 70..130 x 8 expiries = 120 calls.
* ``c2``  4096 Heston surfaces with uneven grids (5..60 strikes x 2..20
          expiries, ln(K/F) ~ U[-0.8, 0.5], T log-uniform in [1/252, 5]y),
          per-surface parameters drawn uniformly (about 1.46M contracts).
* ``c3``  1,048,576 Bates contracts, deep-wing stress: ln(K/F) ~ U[-1.2, 0.7],
          T log-uniform in [1/365, 3]y, calls/puts 50/50, grouped as 4096
          surfaces x 256 contracts sharing one parameter set each (the unit
          of one plain ``batch_bates`` call).  Heston parameters use the
          per-surface uniform ranges of ``c2`` (the fixed parameters of ``c1``
          would not be "drawn"), plus lambda ~ U[0,1.5], mu_j ~ U[-0.3,0.1],
          sigma_j ~ U[0.05,0.4].
* ``c4``  256 Heston calibration surfaces of 30 strikes x 10 expiries.
* ``c5``  the serving request stream (see ``serving_requests``).

Contracts use the C-ABI record (include/ope.h ``ope_contract``, 56 bytes):
spot, strike, expiry, rate, div_yield, vol, opt_type (0 call, 1 put), pad.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

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
    ]
)
assert CONTRACT_DTYPE.itemsize == 56

C1_HESTON = np.array([0.04, 1.5, 0.04, 0.5, -0.7])  # v0, kappa, theta, sigma, rho
TOL_CONFIG = 1e-10  # the configs' absolute GK tolerance


@dataclass
class Workload:
    name: str
    contracts: np.ndarray          # CONTRACT_DTYPE, len n
    params: np.ndarray             # (n_surf, 5) Heston or (n_surf, 8) Bates
    surf_offsets: np.ndarray       # int64, n_surf + 1; surface s owns [off[s], off[s+1])
    bates: bool
    tol: float

    @property
    def n(self) -> int:
        return int(self.contracts.size)

    @property
    def n_surf(self) -> int:
        return int(self.params.shape[0])

    def surf_idx(self) -> np.ndarray:
        counts = np.diff(self.surf_offsets)
        return np.repeat(np.arange(self.n_surf, dtype=np.int32), counts)

    def subset(self, surfaces) -> "Workload":
        """The workload restricted to the given surface indices (in order)."""
        surfaces = np.asarray(surfaces, dtype=np.int64)
        parts = [self.contracts[self.surf_offsets[s]:self.surf_offsets[s + 1]] for s in surfaces]
        counts = [p.size for p in parts]
        off = np.zeros(len(surfaces) + 1, np.int64)
        off[1:] = np.cumsum(counts)
        return Workload(self.name + "-subset", np.concatenate(parts) if parts else self.contracts[:0],
                        self.params[surfaces].copy(), off, self.bates, self.tol)


def _heston_draw(rng: np.random.Generator, n: int) -> np.ndarray:
    v0 = rng.uniform(0.01, 0.2, n)
    kappa = rng.uniform(0.2, 5.0, n)
    theta = rng.uniform(0.01, 0.2, n)
    sigma = rng.uniform(0.1, 1.0, n)
    rho = rng.uniform(-0.95, 0.2, n)
    return np.stack([v0, kappa, theta, sigma, rho], axis=1)


def c1() -> Workload:
    strikes = 70.0 + 60.0 * np.arange(15) / 14.0
    expiries = np.array([0.05, 0.1, 0.25, 0.5, 0.75, 1.0, 1.5, 2.0])
    T, K = np.meshgrid(expiries, strikes, indexing="ij")
    con = np.zeros(T.size, CONTRACT_DTYPE)
    con["spot"], con["strike"], con["expiry"] = 100.0, K.ravel(), T.ravel()
    con["rate"], con["div_yield"], con["vol"], con["opt_type"] = 0.03, 0.01, 0.2, 0
    return Workload("c1-heston-surface-120", con, C1_HESTON[None, :].copy(),
                    np.array([0, con.size], np.int64), False, TOL_CONFIG)


def c2(n_surf: int = 4096, seed: int = 2) -> Workload:
    rng = np.random.default_rng(seed)
    params = _heston_draw(rng, n_surf)
    rates = rng.uniform(0.0, 0.06, n_surf)
    divs = rng.uniform(0.0, 0.03, n_surf)
    parts, off = [], [0]
    for s in range(n_surf):
        nk = int(rng.integers(5, 61))
        nt = int(rng.integers(2, 21))
        T = np.sort(np.exp(rng.uniform(np.log(1 / 252), np.log(5.0), nt)))
        m = np.sort(rng.uniform(-0.8, 0.5, nk))
        TT, MM = np.meshgrid(T, m, indexing="ij")
        F = 100.0 * np.exp((rates[s] - divs[s]) * TT)
        con = np.zeros(TT.size, CONTRACT_DTYPE)
        con["spot"], con["strike"], con["expiry"] = 100.0, (F * np.exp(MM)).ravel(), TT.ravel()
        con["rate"], con["div_yield"], con["vol"] = rates[s], divs[s], 0.2
        con["opt_type"] = rng.integers(0, 2, TT.size)
        parts.append(con)
        off.append(off[-1] + con.size)
    return Workload("c2-heston-4096-surfaces", np.concatenate(parts), params,
                    np.array(off, np.int64), False, TOL_CONFIG)


def c3(n: int = 1 << 20, per_surface: int = 256, seed: int = 3) -> Workload:
    rng = np.random.default_rng(seed)
    n_surf = (n + per_surface - 1) // per_surface
    h = _heston_draw(rng, n_surf)
    lam = rng.uniform(0.0, 1.5, n_surf)
    mu_j = rng.uniform(-0.3, 0.1, n_surf)
    sig_j = rng.uniform(0.05, 0.4, n_surf)
    params = np.concatenate([h, lam[:, None], mu_j[:, None], sig_j[:, None]], axis=1)
    rates = rng.uniform(0.0, 0.06, n_surf)
    divs = rng.uniform(0.0, 0.03, n_surf)
    off = np.minimum(np.arange(n_surf + 1, dtype=np.int64) * per_surface, n)
    sidx = np.repeat(np.arange(n_surf), np.diff(off))
    T = np.exp(rng.uniform(np.log(1 / 365), np.log(3.0), n))
    m = rng.uniform(-1.2, 0.7, n)
    r, q = rates[sidx], divs[sidx]
    con = np.zeros(n, CONTRACT_DTYPE)
    con["spot"] = 100.0
    con["strike"] = 100.0 * np.exp((r - q) * T) * np.exp(m)
    con["expiry"], con["rate"], con["div_yield"], con["vol"] = T, r, q, 0.2
    con["opt_type"] = rng.integers(0, 2, n)
    return Workload(f"c3-bates-deepwing-{n}", con, params, off, True, TOL_CONFIG)


def feller_heston_draw(rng: np.random.Generator, n: int) -> np.ndarray:
    """Heston parameters from the c2 ranges, rejection-sampled to 2*kappa*theta > sigma^2."""
    out = np.zeros((0, 5))
    while out.shape[0] < n:
        d = _heston_draw(rng, 4 * n)
        ok = 2.0 * d[:, 1] * d[:, 2] > d[:, 3] ** 2
        out = np.concatenate([out, d[ok]])
    return out[:n]


def c4_grid(n_surf: int = 256, n_k: int = 30, n_t: int = 10, seed: int = 4):
    """Calibration quote grids: returns (contracts, offsets, true_params, rates, divs)."""
    rng = np.random.default_rng(seed)
    true_p = feller_heston_draw(rng, n_surf)
    rates = rng.uniform(0.0, 0.06, n_surf)
    divs = rng.uniform(0.0, 0.03, n_surf)
    parts, off = [], [0]
    for s in range(n_surf):
        T = np.exp(np.linspace(np.log(0.1), np.log(3.0), n_t))
        m = np.linspace(-0.4, 0.3, n_k)
        TT, MM = np.meshgrid(T, m, indexing="ij")
        F = 100.0 * np.exp((rates[s] - divs[s]) * TT)
        K = F * np.exp(MM)
        con = np.zeros(TT.size, CONTRACT_DTYPE)
        con["spot"], con["strike"], con["expiry"] = 100.0, K.ravel(), TT.ravel()
        con["rate"], con["div_yield"], con["vol"] = rates[s], divs[s], 0.2
        con["opt_type"] = np.where(MM.ravel() >= 0.0, 0, 1)  # OTM side: calls above F, puts below
        parts.append(con)
        off.append(off[-1] + con.size)
    return np.concatenate(parts), np.array(off, np.int64), true_p, rates, divs


def by_name(name: str) -> Workload:
    return {"c1": c1, "c2": c2, "c3": c3}[name]()


def c4(price_fn, iv_fn, n_surf: int = 256, n_k: int = 30, n_t: int = 10, seed: int = 4, noise: float = 0.005):
    """Config 4 calibration problems: quotes priced from seeded true Heston
    parameters (Feller-satisfying draws from the c2 ranges), inverted to IV,
    perturbed by N(0, noise) IV noise; start points truth x U(0.7, 1.3).

    price_fn(contracts, params, surf_idx) -> prices; iv_fn(contracts, prices) -> (iv, ok).
    Quotes whose model IV cannot be inverted or falls outside (0.01, 2) are
    dropped, as the reference's quote builder does (calibration.rs:993-995).
    Returns (quotes, iv_market, offsets, true_params, p0).
    """
    con, off, true_p, _, _ = c4_grid(n_surf, n_k, n_t, seed)
    sidx = np.repeat(np.arange(n_surf, dtype=np.int32), np.diff(off))
    px = price_fn(con, true_p, sidx)
    iv, ok = iv_fn(con, px)
    ok = ok & (iv > 0.01) & (iv < 2.0)
    rng = np.random.default_rng(seed + 1000)
    iv_mkt = np.maximum(iv + rng.normal(0.0, noise, iv.size), 1e-3)
    keep = np.where(ok)[0]
    counts = np.bincount(sidx[keep], minlength=n_surf)
    new_off = np.zeros(n_surf + 1, np.int64)
    new_off[1:] = np.cumsum(counts)
    p0 = true_p * rng.uniform(0.7, 1.3, true_p.shape)
    return con[keep], iv_mkt[keep], new_off, true_p, p0
