"""Write tests/golden/ref_inputs.txt: the contracts on which the reference
crate's own prices pin the oracle (oracle/ref_golden/make_ref_golden.sh runs
the reference on them where cargo exists).  Config 1 (120 Heston calls), a
256-contract sample of the Bates deep-wing batch (puts and calls), and the
twelve corner contracts of corner_cap_contracts.json -- all at the
reference's own quadrature tolerance, 1e-8 (heston.rs:228).  Floats are
written in Python's shortest round-trip form, which Rust parses exactly.

Run from the repository root:  python tests/golden/make_ref_inputs.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "options-pricing-engine-rs_b200")]


def rows():
    from ope_b200 import workloads as W

    out = []
    w1 = W.c1()
    for c in w1.contracts:
        out.append(("heston", list(w1.params[0]), c))
    w3 = W.c3(n=4096, per_surface=256)
    rng = np.random.default_rng(3)
    si = w3.surf_idx()
    for i in np.sort(rng.choice(w3.n, 256, replace=False)):
        out.append(("bates", list(w3.params[si[i]]), w3.contracts[i]))
    with open(os.path.join(HERE, "corner_cap_contracts.json")) as f:
        for e in json.load(f)["contracts"]:
            c = np.zeros(1, W.CONTRACT_DTYPE)[0]
            for k, v in e["contract"].items():
                c[k] = float.fromhex(v)
            c["opt_type"] = e["opt_type"]
            out.append(("bates" if e["bates"] else "heston", [float.fromhex(x) for x in e["params"]], c))
    return out


def main() -> None:
    lines = ["# model params ; spot strike expiry rate div_yield call|put   (tol 1e-8)"]
    for model, p, c in rows():
        lines.append(f"{model} {' '.join(repr(float(x)) for x in p)} ; "
                     + " ".join(repr(float(c[k])) for k in ("spot", "strike", "expiry", "rate", "div_yield"))
                     + (" put" if int(c["opt_type"]) == 1 else " call"))
    with open(os.path.join(HERE, "ref_inputs.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
