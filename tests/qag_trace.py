"""Comparison of two step traces of the greedy GK15 quadrature
(heston.rs:193-212, adaptive_gk): the device library's (ope_b200.trace_integral,
the pricing kernel's own warp routine) and the oracle's (oracle.trace_integral).

Both record, per step j (0 = the first panel [0, 1], j >= 1 = the j-th
bisection): a, b, ew of the bisected panel; kl, el, kr, er of its children;
the running error and total; the 15 integrand values of the left child and the
15 of the right child.  Panel geometry is computed bit-identically on both
sides, so while both make the same choices the live lists hold the same
panels, and each panel's K, error estimate and node values can be compared
side by side.  Where a choice differs, the two error estimates that decided it
show whether it was a near tie.
"""
from __future__ import annotations

import math

import numpy as np

A, B, EW, KL, EL, KR, ER, ERR, TOTAL = range(9)
F_LEFT, F_RIGHT = slice(9, 24), slice(24, 39)


def panels_before(tr: np.ndarray, k: int) -> dict:
    """The live panels before step k (k >= 1): {(a, b): (K, err, 15 node values)}."""
    live = {(0.0, 1.0): (tr[0, KL], tr[0, EL], tr[0, F_LEFT])}
    for j in range(1, k):
        a, b = tr[j, A], tr[j, B]
        del live[(a, b)]
        m = 0.5 * (a + b)
        live[(a, m)] = (tr[j, KL], tr[j, EL], tr[j, F_LEFT])
        live[(m, b)] = (tr[j, KR], tr[j, ER], tr[j, F_RIGHT])
    return live


def first_divergence(dev: np.ndarray, orc: np.ndarray):
    """First step whose bisected panel differs, or where one side stopped and
    the other went on; None if the two traces make the same choices."""
    n = min(len(dev), len(orc))
    for j in range(1, n):
        if dev[j, A] != orc[j, A] or dev[j, B] != orc[j, B]:
            return j
    return None if len(dev) == len(orc) else n


def _ulps(x: float, y: float) -> float:
    return abs(x - y) / max(math.ulp(abs(y)), 5e-324)


def node_agreement(dev: np.ndarray, orc: np.ndarray, upto: int) -> float:
    """Worst |f_dev - f_orc| over the steps before `upto`, relative to the
    largest |f| of the same step's 30 values (the scale of the sums formed
    from them)."""
    worst = 0.0
    for j in range(upto):
        fd, fo = dev[j, 9:], orc[j, 9:]
        scale = np.max(np.abs(fo))
        if scale > 0:
            worst = max(worst, float(np.max(np.abs(fd - fo)) / scale))
    return worst


def divergence_report(dev: np.ndarray, orc: np.ndarray) -> dict | None:
    """Where and why the two traces part.  For a different choice at step k:
    the device bisected panel P_dev, the oracle P_orc; their error estimates on
    each side, each side's relative margin between the two, how far the two
    sides' estimates of the same panel lie apart (relative, and in ulps), and
    how closely the node values agreed up to k."""
    k = first_divergence(dev, orc)
    if k is None:
        return None
    rep = {"step": k, "steps_dev": len(dev), "steps_orc": len(orc),
           "node_rel_before": node_agreement(dev, orc, k)}
    if k >= min(len(dev), len(orc)):
        # one side stopped (err <= tol or the 200-panel cap), the other did not
        rep.update(kind="stop", err_dev=float(dev[k - 1, ERR]), err_orc=float(orc[k - 1, ERR]))
        return rep
    ld, lo = panels_before(dev, k), panels_before(orc, k)
    pd = (dev[k, A], dev[k, B])
    po = (orc[k, A], orc[k, B])
    ed = {p: ld[p][1] for p in (pd, po)}
    eo = {p: lo[p][1] for p in (pd, po)}
    rep.update(
        kind="choice",
        panel_dev=pd, panel_orc=po,
        err_dev=(float(ed[pd]), float(ed[po])),  # device's estimates of (P_dev, P_orc)
        err_orc=(float(eo[pd]), float(eo[po])),  # oracle's estimates of (P_dev, P_orc)
        margin_dev=float((ed[pd] - ed[po]) / ed[pd]) if ed[pd] > 0 else 0.0,
        margin_orc=float((eo[po] - eo[pd]) / eo[po]) if eo[po] > 0 else 0.0,
        err_rel_diff=max(float(abs(ed[p] - eo[p]) / eo[p]) if eo[p] > 0 else float(ed[p] != eo[p]) for p in (pd, po)),
        err_ulps=max(_ulps(ed[p], eo[p]) for p in (pd, po)),
        k_rel_diff=max(float(abs(ld[p][0] - lo[p][0]) / max(abs(lo[p][0]), 5e-324)) for p in (pd, po)),
    )
    return rep


def final_error(tr: np.ndarray) -> float:
    """The quadrature's own error estimate when it stopped."""
    return float(tr[-1, ERR])


def price_bound(c, e1: float, e2: float) -> float:
    """Largest price difference two quadratures whose integrals each lie within
    their own error estimates of the exact ones can show: e1, e2 are the SUMS
    of the two sides' final error estimates of P1 and P2.  price = S e^{-qT}
    (1/2 + I1/pi) - K e^{-rT} (1/2 + I2/pi) (heston.rs:95-98); the max(., 0)
    clamp and put-call parity (heston.rs:70) do not enlarge a difference."""
    s, k, t, r, q = (float(c[f]) for f in ("spot", "strike", "expiry", "rate", "div_yield"))
    return (s * math.exp(-q * t) * e1 + k * math.exp(-r * t) * e2) / math.pi
