"""Generate the committed golden fixtures under tests/golden/.

1. mpmath_prices.json — independent high-precision known answers: the
   reference's Gil-Pelaez formula (heston.rs:82-127, bates.rs:49-83: the
   Albrecher stable CF with drift r, the P1 normaliser CF(-i), the call
   clamped at 0 and the put by parity) evaluated with mpmath at 40 digits and
   mpmath's own tanh-sinh quadrature on [0, inf) — no Gauss-Kronrod, no
   panels, nothing shared with the oracle or the CUDA path.  Each value is
   computed twice (two different interval splittings) and kept only if they
   agree to 1e-20.
2. csqrt_sweep.json — principal square roots for the reference's
   fast_csqrt sweep (heston.rs:255-307): the same magnitude x angle grid,
   near-axis angles and axis points, with mpmath's principal sqrt.
3. oracle_c1.json / oracle_bates_grid.json — the oracle's prices at
   tol = 1e-10 on config 1 and on the reference's Bates arbitrage grid
   (bates.rs:147-173), pinned so later oracle edits cannot drift silently.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import mpmath as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "options-pricing-engine-rs_b200"))

mp.mp.dps = 40
I = mp.mpc(0, 1)


def stable_cf(phi, t, r, p):
    v0, kappa, theta, sigma, rho = [mp.mpf(x) for x in p]
    xi = kappa - rho * sigma * phi * I
    d = mp.sqrt(xi * xi + sigma * sigma * phi * (phi + I))
    g = (xi - d) / (xi + d)
    edt = mp.exp(-d * t)
    a = (g * edt - 1) / (g - 1)
    c = (kappa * theta / (sigma * sigma)) * ((xi - d) * t - 2 * mp.log(a))
    dd = v0 * (xi - d) * (1 - edt) / (sigma * sigma * (1 - g * edt))
    return mp.exp(r * phi * I * t + c + dd)


def jump_cf(phi, t, lam, mu_j, sigma_j):
    lam, mu_j, sigma_j = mp.mpf(lam), mp.mpf(mu_j), mp.mpf(sigma_j)
    comp = mp.exp(mu_j + sigma_j * sigma_j / 2) - 1
    jump = mp.exp(phi * I * mu_j - phi * phi * sigma_j * sigma_j / 2)
    return mp.exp(lam * t * (jump - 1 - I * phi * comp))


def price(s, k, t, r, q, p, opt, splits):
    s, k, t, r, q = [mp.mpf(x) for x in (s, k, t, r, q)]
    x = mp.log(s / k)
    bates = len(p) == 8

    def cf(phi):
        v = stable_cf(phi, t, r, p[:5])
        if bates:
            v *= jump_cf(phi, t, *p[5:])
        return v

    cf_mi = cf(mp.mpc(0, -1))
    f1 = lambda u: mp.re(mp.exp(I * u * x) * cf(mp.mpc(u, -1)) / cf_mi / (I * u))  # noqa: E731
    f2 = lambda u: mp.re(mp.exp(I * u * x) * cf(mp.mpc(u, 0)) / (I * u))  # noqa: E731
    i1 = mp.quad(f1, splits)
    i2 = mp.quad(f2, splits)
    p1 = mp.mpf(1) / 2 + i1 / mp.pi
    p2 = mp.mpf(1) / 2 + i2 / mp.pi
    call = max(s * mp.exp(-q * t) * p1 - k * mp.exp(-r * t) * p2, mp.mpf(0))
    return call if opt == 0 else call - s * mp.exp(-q * t) + k * mp.exp(-r * t)


def mpmath_cases():
    hp = [0.04, 2.0, 0.04, 0.3, -0.7]          # heston.rs:236-239
    hp2 = [0.09, 1.0, 0.09, 0.8, -0.5]         # heston.rs:386
    c1p = [0.04, 1.5, 0.04, 0.5, -0.7]         # config 1
    bp = hp + [0.5, -0.1, 0.15]                # bates.rs:94-96
    bp2 = hp2 + [1.0, -0.2, 0.25]              # bates.rs:151-154
    cases = []
    for p in (hp, hp2, c1p):
        for t in (0.25, 1.0, 2.0):
            for k in (80.0, 100.0, 120.0):
                for opt in (0, 1):
                    cases.append((100.0, k, t, 0.03, 0.01, p, opt))
    for p in (bp, bp2):
        for t in (0.25, 1.0):
            for k in (85.0, 100.0, 115.0):
                cases.append((100.0, k, t, 0.05, 0.0, p, 0))
    return cases


def make_mpmath():
    out = []
    s1 = [0, 0.5, 2, 5, 10, 20, 40, 80, 160, mp.inf]
    s2 = [0, 1, 3, 7, 15, 30, 60, 120, 250, mp.inf]
    for (s, k, t, r, q, p, opt) in mpmath_cases():
        a = price(s, k, t, r, q, p, opt, s1)
        b = price(s, k, t, r, q, p, opt, s2)
        if abs(a - b) > mp.mpf("1e-20"):
            print("skip (quadrature disagreement)", s, k, t, p, opt, mp.nstr(a - b, 5))
            continue
        out.append({"spot": s, "strike": k, "expiry": t, "rate": r, "div_yield": q, "params": p,
                    "opt_type": opt, "price": mp.nstr(a, 25)})
        print(len(out), k, t, opt, mp.nstr(a, 18))
    with open(os.path.join(HERE, "mpmath_prices.json"), "w") as f:
        json.dump(out, f, indent=1)


def make_csqrt():
    mags = [1e-6, 1e-3, 0.1, 1.0, 10.0, 100.0, 1e4, 1e6]
    n = 37
    angles = [-mp.pi + 2 * mp.pi * i / (n - 1) for i in range(n)]
    for tiny in (1e-2, 1e-4, 1e-6, 1e-8, 1e-10, 1e-12):
        for base in (mp.mpf(0), mp.pi, mp.pi / 2, -mp.pi / 2):
            angles.append(base + tiny)
            angles.append(base - tiny)
    pts = []
    for mag in mags:
        for ang in angles:
            z = mp.mpc(float(mag * mp.cos(ang)), float(mag * mp.sin(ang)))  # the double-rounded input
            pts.append(z)
    for re, im in ((4.0, 0.0), (-4.0, 0.0), (0.0, 4.0), (0.0, -4.0), (0.0, 0.0)):
        pts.append(mp.mpc(re, im))
    # heston.rs:298-304 regression point: 1 + 1e-8 * (0.5 - i) * ((0.5 - i) + i)
    w = mp.mpc(0.5, -1.0)
    reg = 1.0 + complex(1e-8 * complex(w) * (complex(w) + 1j))
    pts.append(mp.mpc(reg.real, reg.imag))
    out = []
    for z in pts:
        sq = mp.sqrt(z)
        out.append([float(z.real), float(z.imag), mp.nstr(sq.real, 25), mp.nstr(sq.imag, 25)])
    with open(os.path.join(HERE, "csqrt_sweep.json"), "w") as f:
        json.dump(out, f)


def make_oracle_fixtures():
    import numpy as np

    from ope_b200 import workloads as W
    from oracle import oracle as O

    O.build()
    w = W.c1()
    px = O.batch_price(w.contracts, w.params, False, w.tol)
    with open(os.path.join(HERE, "oracle_c1.json"), "w") as f:
        json.dump({"tol": w.tol, "params": w.params[0].tolist(),
                   "strike": w.contracts["strike"].tolist(), "expiry": w.contracts["expiry"].tolist(),
                   "price": [float.hex(float(v)) for v in px]}, f, indent=0)
    sets = [[0.04, 2.0, 0.04, 0.3, -0.7, 0.5, -0.1, 0.15], [0.09, 1.0, 0.09, 0.8, -0.5, 1.0, -0.2, 0.25]]
    rows = []
    for p in sets:
        for t in (0.02, 0.1, 0.25, 0.5, 1.0, 2.0):
            for k in (70.0, 85.0, 100.0, 115.0, 130.0, 150.0, 200.0):
                v = O.bates_price(100.0, k, t, 0.03, 0.0, p, 0, 1e-10)
                rows.append({"params": p, "expiry": t, "strike": k, "price": float.hex(float(v))})
    with open(os.path.join(HERE, "oracle_bates_grid.json"), "w") as f:
        json.dump(rows, f, indent=0)
    print("oracle fixtures:", len(px), len(rows), np.max(px))


if __name__ == "__main__":
    what = sys.argv[1:] or ["csqrt", "oracle", "mpmath"]
    if "csqrt" in what:
        make_csqrt()
    if "oracle" in what:
        make_oracle_fixtures()
    if "mpmath" in what:
        make_mpmath()
