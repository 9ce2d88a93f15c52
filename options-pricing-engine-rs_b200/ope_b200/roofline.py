"""Algorithmic FP64 work of the pricing path (the roofline numerator).

Unit of work: one GK15 node evaluation, i.e. one call of gk_integrate's g(t)
(heston.rs:221-227) with its cf_integrand / bates_integrand (heston.rs:101-109,
bates.rs:65-73), stable_cf (heston.rs:113-127), fast_csqrt (heston.rs:155-175),
jump_cf (bates.rs:77-83) and its share of the panel sums (heston.rs:180-187).

F_node is tallied operation by operation from the REFERENCE's formulation
(not from the CUDA kernel, which merges exponentials and so does less), with
this frozen cost table, in FP64 operations:

    add/sub/mul = 1, div = 4, sqrt = 4, hypot = 8,
    exp = 16, log = 16, sin = 16, cos = 16, atan2 = 24

An FMA counts as its add and its mul (2), the same convention as the
measured DFMA peak (2 flops per DFMA) it is divided by.  Work per contract =
sum over its two integrals of nodes * F_node(integral), with
nodes = 15 * (1 + 2 * bisections) (heston.rs:195, 204-205).
"""
from __future__ import annotations

import numpy as np

COST = {"add": 1, "mul": 1, "div": 4, "sqrt": 4, "hypot": 8, "exp": 16, "log": 16, "sin": 16, "cos": 16,
        "atan2": 24}


def _ops(**kw):
    return kw


def _cexp():
    return _ops(exp=1, cos=1, sin=1, mul=2)


def _cmul():
    return _ops(mul=4, add=2)


def _cdiv():
    return _ops(mul=6, add=3, div=2)


def _sum(*parts):
    out: dict = {}
    for p in parts:
        for k, v in p.items():
            out[k] = out.get(k, 0) + v
    return out


def stable_cf_ops():
    """heston.rs:113-127 at a complex phi, operation by operation."""
    xi = _sum(_ops(mul=1), _ops(mul=2), _cmul(), _ops(add=2))            # kappa - rho*sigma*phi*i
    z = _sum(_cmul(), _ops(mul=1), _ops(mul=2), _ops(add=2), _cmul(), _ops(add=2))  # xi^2 + s^2 phi (phi+i)
    csqrt = _ops(hypot=1, add=1, div=2, sqrt=1, mul=1)                     # heston.rs:165-169
    g = _sum(_ops(add=4), _cdiv())
    edt = _sum(_ops(mul=2), _cexp())
    a = _sum(_cmul(), _ops(add=2), _cdiv())
    c = _sum(_ops(mul=2, div=1), _ops(add=2, mul=2), _ops(hypot=1, log=1, atan2=1), _ops(mul=2, add=2),
             _ops(mul=2))
    dd = _sum(_ops(add=2, mul=2), _ops(add=2), _cmul(), _ops(mul=1), _cmul(), _ops(add=2), _ops(mul=2), _cdiv())
    fin = _sum(_ops(mul=2), _cmul(), _ops(mul=2), _ops(add=4), _cexp())
    return _sum(xi, z, csqrt, g, edt, a, c, dd, fin)


def jump_cf_ops():
    """bates.rs:77-83 (comp is per node in the reference, counted here too)."""
    comp = _ops(exp=1, mul=2, add=2)
    jump = _sum(_cmul(), _ops(mul=2), _ops(mul=2), _cmul(), _ops(mul=4), _ops(add=2), _cexp())
    outer = _sum(_ops(add=1), _cmul(), _ops(mul=2), _ops(add=2), _ops(mul=3), _cexp())
    return _sum(comp, jump, outer)


def node_ops(bates: bool, p1: bool):
    integrand = _sum(stable_cf_ops(), jump_cf_ops() if bates else {}, _cmul() if bates else {},
                     _cdiv() if p1 else {},                                  # cf /= cf_mi
                     _ops(mul=1), _cexp(), _cmul(), _cdiv())                 # e^{iux} cf / (iu)
    subst = _ops(add=1, div=2, mul=1)                                        # (1-t)/t, f/(t*t)
    panel = _ops(mul=1, add=1)                                               # c + h*x_i
    sums = _ops(mul=2, add=2)                                                # K15 term + G7 share (rounded up)
    return _sum(integrand, subst, panel, sums)


def f_node(bates: bool, p1: bool) -> int:
    return int(sum(COST[k] * v for k, v in node_ops(bates, p1).items()))


F_NODE = {(b, p): f_node(b, p) for b in (False, True) for p in (True, False)}


def work_flops(bisections: np.ndarray, bates: bool) -> float:
    """Total FP64 ops for contracts with per-integral bisection counts (n, 2): [P1, P2]."""
    nb = np.asarray(bisections, dtype=np.int64).reshape(-1, 2)
    nodes = 15 * (1 + 2 * nb)
    return float(nodes[:, 0].sum() * F_NODE[(bates, True)] + nodes[:, 1].sum() * F_NODE[(bates, False)])


def nodes_total(bisections: np.ndarray) -> int:
    nb = np.asarray(bisections, dtype=np.int64)
    return int((15 * (1 + 2 * nb)).sum())


if __name__ == "__main__":
    for (b, p), v in F_NODE.items():
        print(f"bates={b} p1={p}: F_node = {v} FP64 ops")
