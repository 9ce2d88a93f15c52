"""GPU: the bounds-checked build (lib/checked/, make CHECKED=1) runs the
pricing (per contract and the run kernel), gradient, Greeks and calibration
paths with its device invariant checks on -- panel-list indices and counts,
surface indices, panel-list slots, run-cache entries -- and must finish with a zero check word and the same results as the
ordinary build.  (A stand-in for a memory checker, which is not available
on this pool.)"""
import ctypes

import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu

S = 100.0


def _word(L):
    w, checked = ctypes.c_uint32(), ctypes.c_int32()
    assert L.ope_check_word(ctypes.byref(w), ctypes.byref(checked)) == 0
    return w.value, checked.value


def _ok(L, rc):
    assert rc == 0, L.ope_last_error().decode()


def test_checked_build_runs_clean(ope, oracle):
    import os

    if not os.path.exists(ope._lib.CHECKED_LIB_PATH):
        pytest.fail("the bounds-checked build is missing: python __graft_entry__.py build")
    L = ope._lib.open_library(ope._lib.CHECKED_LIB_PATH)
    _, checked = _word(L)
    assert checked == 1
    o = ope._lib.Options(tol=1e-10, flags=0, reserved=0, stream=None)

    # pricing: many surfaces (one persistent launch) and one surface
    w = W.c3(n=4096, per_surface=256, seed=31)
    got = np.zeros(w.n)
    _ok(L, L.ope_price_surfaces(1, w.contracts.ctypes.data, w.n, w.surf_offsets.ctypes.data, w.n_surf,
                                w.params.ctypes.data, got.ctypes.data, ctypes.byref(o)))
    ref = ope.price_surfaces(ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, tol=w.tol)
    assert np.max(np.abs(got - ref)) <= 1e-12 * S
    one = np.zeros(256)
    _ok(L, L.ope_batch_price_ex(1, w.contracts.ctypes.data, 256, w.params[0].ctypes.data, one.ctypes.data,
                                ctypes.byref(o)))
    assert np.max(np.abs(one - ref[:256])) <= 1e-12 * S

    # the run kernel (grid surfaces, 8 contracts per unit: the run cache's
    # entries and child links checked) -- bit-identical to the ordinary build
    g = W.c2(n_surf=120, seed=32)
    E = (ope._lib.TuneEntry * ope._lib.TUNE_CLASSES)()
    for e in E:
        e.shape.warps_per_block, e.shape.occupancy, e.shape.per_unit = 4, 1.0, 8
    _ok(L, L.ope_set_tune_table(0, E))
    gpx = np.zeros(g.n)
    _ok(L, L.ope_price_surfaces(0, g.contracts.ctypes.data, g.n, g.surf_offsets.ctypes.data, g.n_surf,
                                g.params.ctypes.data, gpx.ctypes.data, ctypes.byref(o)))
    pu = ctypes.c_int32()
    _ok(L, L.ope_last_per_unit(ctypes.byref(pu)))
    assert pu.value == 8
    gref = ope.price_surfaces(ope.MODEL_HESTON, g.contracts, g.surf_offsets, g.params, tol=1e-10)
    assert np.array_equal(gpx.view(np.int64), gref.view(np.int64))

    # reverse-mode gradient (panel lists stored by the pricing kernel, read by the backward pass)
    n = 1024
    pg, gg = np.zeros(n), np.zeros((n, 8))
    off = w.surf_offsets[:5].copy()
    _ok(L, L.ope_price_gradient_surfaces(1, w.contracts.ctypes.data, n, off.ctypes.data, 4, w.params.ctypes.data,
                                         pg.ctypes.data, gg.ctypes.data, ctypes.byref(o)))
    rp, rg = ope.price_gradient_surfaces(ope.MODEL_BATES, w.contracts[:n], off, w.params[:4], tol=1e-10)
    assert np.max(np.abs(gg - rg) / (1e-7 * np.abs(rg) + 1e-9 * S)) <= 1.0

    # AD Greeks (pricing with parameter indices + adjoint)
    c1 = W.c1()
    gad = np.zeros(c1.n, dtype=ope.RESULT_DTYPE)
    _ok(L, L.ope_batch_greeks_ad(0, c1.contracts.ctypes.data, c1.n, c1.params[0].ctypes.data, gad.ctypes.data,
                                 ctypes.byref(o)))
    rgad = ope.batch_greeks_ad(ope.MODEL_HESTON, c1.contracts, c1.params[0], tol=1e-10)
    assert np.max(np.abs(gad["price"] - rgad["price"])) <= 1e-12 * S

    # calibration (two panel-list slots per surface) and multistart (restart groups)
    rows, ivs = [], []
    for t in (0.25, 0.5, 1.0):
        for k in (80.0, 90.0, 95.0, 100.0, 105.0, 110.0, 120.0):
            ot = 0 if k >= 100.0 else 1
            px = oracle.heston_price(100.0, k, t, 0.03, 0.0, [0.04, 2.0, 0.04, 0.3, -0.5], ot)
            c = oracle.contracts(100.0, k, t, 0.03, 0.0, ot)
            iv = oracle.implied_vol(c, px)
            if iv is not None and 0.01 < iv < 2.0:
                rows.append(c[0])
                ivs.append(iv)
    con, iv = np.array(rows), np.array(ivs)
    qoff = np.array([0, iv.size], dtype=np.int64)
    p0 = np.array([0.05, 1.5, 0.05, 0.4, -0.3])
    out = np.zeros(1, dtype=ope.CALIB_RESULT_DTYPE)
    oc = ope._lib.Options(tol=1e-8, flags=0, reserved=0, stream=None)
    _ok(L, L.ope_calibrate_surfaces(0, con.ctypes.data, iv.ctypes.data, None, iv.size, qoff.ctypes.data, 1,
                                    p0.ctypes.data, out.ctypes.data, ctypes.byref(oc)))
    r = ope.calibrate_heston(con, iv, p0)
    assert out[0]["converged"] == r["converged"] and abs(out[0]["rmse"] - r["rmse"]) < 1e-10
    ms = np.zeros(1, dtype=ope.MULTISTART_RESULT_DTYPE)
    bad = np.array([0.25, 6.0, 0.3, 0.15, 0.6])
    _ok(L, L.ope_calibrate_multistart(0, con.ctypes.data, iv.ctypes.data, None, iv.size, qoff.ctypes.data, 1,
                                      bad.ctypes.data, 8, 12345, None, ms.ctypes.data, None, ctypes.byref(oc)))
    rm = ope.calibrate_heston_multistart(con, iv, bad, 8, 12345)
    assert ms[0]["best_restart"] == rm["best_restart"] and abs(ms[0]["best"]["rmse"] - rm["best"]["rmse"]) < 1e-10

    word, _ = _word(L)
    assert word == 0, f"device check word {word:#x}"
