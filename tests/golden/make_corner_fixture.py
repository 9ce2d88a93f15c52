"""Generate tests/golden/corner_cap_contracts.json: the twelve contracts of a
240,000-contract corner sample (12 draws of 20,000 at tol 1e-12) on which an
earlier build of the device kernels differed most from the oracle -- four of
them by more than the 1e-9 S parity bar.  All have both integrals at the
200-panel cap of heston.rs:194 with expiries down to 1e-4 years, log-moneyness
near +-4 and v0 down to 1e-6, so the integrands' phase u ln(S/K) reaches 1e7:
there one ulp of u, of ln(S/K) or of the summed phase moves a node value by
1e-9 relative.

The draw is the one of tests/test_gpu_fuzz.py (`_draw`), widened to those
corners; the (model, draw, index) triples were found by comparing the device
with the oracle over the whole sample.  Each fixture entry keeps the contract
and parameters bit-exactly (hex) and the oracle's price and bisection counts
at tol 1e-12, so later oracle edits cannot drift silently.

Run from the repository root:  python tests/golden/make_corner_fixture.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "options-pricing-engine-rs_b200"), os.path.dirname(HERE)]

S = 100.0
TOL = 1e-12
# (bates, draw, index) of the contracts, worst first
PICKS = [(0, 2, 18318), (1, 2, 18130), (1, 5, 15506), (0, 1, 3548), (0, 3, 2865), (0, 3, 13511),
         (1, 2, 13769), (1, 1, 1714), (0, 5, 9779), (1, 3, 7241), (1, 0, 17573), (1, 2, 17885)]


def corner_draw(bates: bool, draw: int):
    """Draw `draw` of the corner sample: 20,000 contracts, one parameter set each."""
    from test_gpu_fuzz import _draw

    rng = np.random.default_rng(90000 + 100 * draw + 10 * int(bates) + 1)
    n = 20000
    con, p = _draw(rng, n, bates)
    con["expiry"] = np.exp(rng.uniform(np.log(1e-4), np.log(10.0), n))
    con["strike"] = S * np.exp(rng.uniform(-4.0, 4.0, n))
    small = rng.random(n) < 0.2
    p[small, 0] = rng.uniform(1e-6, 1e-4, small.sum())
    p[small, 2] = rng.uniform(1e-6, 1e-4, small.sum())
    return con, p


def main() -> None:
    from oracle import oracle as O

    out = []
    for bates, draw, i in PICKS:
        con, p = corner_draw(bool(bates), draw)
        c = con[i: i + 1]
        price, nb = O.batch_price(c, p[i: i + 1], bool(bates), TOL, surf_idx=np.zeros(1, np.int32), stats=True)
        out.append({
            "bates": bates, "draw": draw, "index": i,
            "contract": {f: float(c[f][0]).hex() for f in ("spot", "strike", "expiry", "rate", "div_yield", "vol")},
            "opt_type": int(c["opt_type"][0]),
            "params": [float(x).hex() for x in p[i]],
            "oracle_price": float(price[0]).hex(),
            "oracle_bisections": [int(nb[0]), int(nb[1])],
        })
    with open(os.path.join(HERE, "corner_cap_contracts.json"), "w") as f:
        json.dump({"tol": TOL, "contracts": out}, f, indent=1)


if __name__ == "__main__":
    main()
