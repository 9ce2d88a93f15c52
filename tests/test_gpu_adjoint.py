"""GPU: the reverse-mode adjoint kernel against the oracle's forward-mode AD
(ad.rs:695-731, 882-895 restated) and against central finite differences.

Bar: relative error <= 1e-7 against forward-mode AD on every gradient
component, with an absolute floor of 1e-9 * S for components that are
themselves tiny (deep out-of-the-money / very short expiries), the same
relative-or-absolute convention as ad.rs:1305-1317.
"""
import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu

S = 100.0
REL = 1e-7
ABS = 1e-9 * S
H_REF = [0.04, 2.0, 0.04, 0.3, -0.7]
B_REF = H_REF + [0.5, -0.1, 0.15]


def _assert_close(got, ref, rel=REL, abs_=ABS, what=""):
    err = np.abs(got - ref)
    lim = rel * np.abs(ref) + abs_
    bad = err > lim
    assert not bad.any(), f"{what}: {int(bad.sum())} entries, worst {float((err / lim).max()):.3g}x the bar; " \
                          f"first {np.argwhere(bad)[:4].tolist()}"


def test_heston_gradient_matches_forward_ad_c1(ope, oracle):
    w = W.c1()
    price, grad = ope.price_gradient_surfaces(ope.MODEL_HESTON, w.contracts, w.surf_offsets, w.params, tol=w.tol)
    rp, rg = oracle.batch_price_gradient(w.contracts, w.params, False, w.tol)
    _assert_close(grad, rg, what="c1 heston grad")
    plain = ope.batch_heston(w.contracts, w.params[0], tol=w.tol)
    assert np.max(np.abs(price - plain)) <= 1e-12 * S


def test_bates_gradient_matches_forward_ad_c3_sample(ope, oracle):
    w = W.c3()
    sub = w.subset([5, 777, 2048])
    price, grad = ope.price_gradient_surfaces(ope.MODEL_BATES, sub.contracts, sub.surf_offsets, sub.params,
                                              tol=sub.tol)
    rp, rg = oracle.batch_price_gradient(sub.contracts, sub.params, True, sub.tol, surf_idx=sub.surf_idx())
    _assert_close(grad, rg, what="c3 bates grad")
    assert np.max(np.abs(price - rp)) <= 1e-8  # dual-path price vs primal (ad.rs:1394-1408 bar is 1e-6)


def test_heston_gradient_matches_forward_ad_c2_sample(ope, oracle):
    w = W.c2()
    sub = w.subset([3, 100, 1000, 4000])
    price, grad = ope.price_gradient_surfaces(ope.MODEL_HESTON, sub.contracts, sub.surf_offsets, sub.params,
                                              tol=sub.tol)
    rp, rg = oracle.batch_price_gradient(sub.contracts, sub.params, False, sub.tol, surf_idx=sub.surf_idx())
    _assert_close(grad, rg, what="c2 heston grad")


@pytest.mark.parametrize("bates", [False, True])
def test_gradient_matches_finite_differences(ope, bates):
    """Fourth-order central differences of the GPU pricer itself (tol 1e-13)."""
    p0 = np.array(B_REF if bates else H_REF)
    model = ope.MODEL_BATES if bates else ope.MODEL_HESTON
    con = np.zeros(6, W.CONTRACT_DTYPE)
    con["spot"], con["strike"] = 100.0, [80.0, 95.0, 100.0, 105.0, 120.0, 100.0]
    con["expiry"], con["rate"], con["div_yield"] = [0.5, 1.0, 1.0, 1.0, 2.0, 0.25], 0.03, 0.01
    con["opt_type"] = [1, 1, 0, 0, 0, 1]
    off = np.array([0, con.size])
    tol = 1e-13
    _, grad = ope.price_gradient_surfaces(model, con, off, p0[None], tol=tol)
    for k in range(p0.size):
        h = 1e-3 * max(abs(p0[k]), 0.05)
        vals = []
        for m in (2, 1, -1, -2):
            p = p0.copy()
            p[k] += m * h
            vals.append(ope.price_surfaces(model, con, off, p[None], tol=tol))
        fd = (-vals[0] + 8 * vals[1] - 8 * vals[2] + vals[3]) / (12 * h)
        _assert_close(grad[:, k], fd, rel=1e-6, abs_=1e-6, what=f"fd param {k}")


def test_jump_sensitivities_signs(ope):  # ad.rs:1022-1027: d price / d mu_j < 0 here
    con = np.zeros(1, W.CONTRACT_DTYPE)
    con["spot"], con["strike"], con["expiry"], con["rate"] = 100.0, 100.0, 1.0, 0.05
    _, g = ope.price_gradient_surfaces(ope.MODEL_BATES, con, [0, 1], np.array([B_REF]))
    assert g[0, 6] < 0.0
    assert g[0, 0] > 0.0  # vega in variance units is positive for a call


def test_gradient_puts_equal_calls(ope):  # ad.rs:726-729: parity terms do not depend on the params
    con = np.zeros(2, W.CONTRACT_DTYPE)
    con["spot"], con["strike"], con["expiry"], con["rate"], con["div_yield"] = 100.0, 110.0, 0.7, 0.02, 0.01
    con["opt_type"] = [0, 1]
    _, g = ope.price_gradient_surfaces(ope.MODEL_BATES, con, [0, 2], np.array([B_REF]), tol=1e-10)
    assert np.array_equal(g[0], g[1])


def test_long_integrals_split_into_chunks_match_forward_ad(ope, oracle):
    """The backward pass splits an integral's stored panels into chunks of 64
    worked by different warps and adds the chunks' partial sums in order;
    contracts whose integrals need more than 64 (and more than 128) final
    panels must match forward-mode AD like any other, alone and inside a
    batch, and give the same gradient either way."""
    w = W.c3(n=1 << 14, per_surface=256, seed=9)
    nb = np.zeros(2 * w.n, np.int32)
    ope.price_surfaces(ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, tol=w.tol, bisections=nb)
    deepest = np.max(nb.reshape(-1, 2), axis=1)
    pick = np.argsort(-deepest)[:24]
    assert deepest[pick[0]] >= 128 and deepest[pick[-1]] >= 64, (deepest[pick[0]], deepest[pick[-1]])
    pick = np.sort(pick)
    sidx = w.surf_idx()[pick]
    con = w.contracts[pick]
    off = np.arange(pick.size + 1, dtype=np.int64)
    par = w.params[sidx]
    price, grad = ope.price_gradient_surfaces(ope.MODEL_BATES, con, off, par, tol=w.tol)
    rp, rg = oracle.batch_price_gradient(con, par, True, w.tol, surf_idx=np.arange(pick.size, dtype=np.int32))
    _assert_close(grad, rg, what="multi-chunk bates grad")
    # the same contracts inside their full surfaces
    _, gfull = ope.price_gradient_surfaces(ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, tol=w.tol)
    assert np.array_equal(gfull[pick], grad)
