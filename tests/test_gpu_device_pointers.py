"""GPU: the ABI's device-pointer mode (OPE_FLAG_DEVICE_PTRS): inputs and
outputs in device memory, work enqueued on the caller's stream.  Every entry
point that supports it runs on a non-default torch stream and must give the
host-pointer path's results bit for bit."""
import ctypes

import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(ope):
    import torch

    st = torch.cuda.Stream()
    lib = ope._lib.load()

    def opts(tol):
        return ope._lib.Options(tol=tol, flags=ope._lib.FLAG_DEVICE_PTRS, reserved=0, stream=st.cuda_stream)

    def dev(a):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(np.uint8).copy()).cuda()

    def host(t, dtype, shape):
        torch.cuda.synchronize()
        return t.cpu().numpy().view(dtype).reshape(shape)

    return torch, st, lib, opts, dev, host


def _ok(ope, rc):
    if rc != 0:
        raise ope.OpeError(rc, ope._lib.load().ope_last_error().decode())


def test_pricing_and_greeks(ope, env):
    torch, st, lib, opts, dev, host = env
    w = W.c3(n=8192, per_surface=256, seed=41)
    o = opts(w.tol)
    d_con, d_off, d_par = dev(w.contracts), dev(w.surf_offsets), dev(w.params)
    d_out = torch.empty(w.n * 8, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(st):
        _ok(ope, lib.ope_price_surfaces(1, d_con.data_ptr(), w.n, d_off.data_ptr(), w.n_surf, d_par.data_ptr(),
                                        d_out.data_ptr(), ctypes.byref(o)))
    got = host(d_out, np.float64, (w.n,))
    assert np.array_equal(got, ope.price_surfaces(ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, tol=w.tol))
    # one parameter set: prices, bump Greeks, AD Greeks
    n = 256
    d_p0 = dev(w.params[0])
    d_px = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    d_gr = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    d_ga = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(st):
        _ok(ope, lib.ope_batch_price_ex(1, d_con.data_ptr(), n, d_p0.data_ptr(), d_px.data_ptr(), ctypes.byref(o)))
        _ok(ope, lib.ope_batch_greeks_ex(1, d_con.data_ptr(), n, d_p0.data_ptr(), d_gr.data_ptr(), ctypes.byref(o)))
        _ok(ope, lib.ope_batch_greeks_ad(1, d_con.data_ptr(), n, d_p0.data_ptr(), d_ga.data_ptr(), ctypes.byref(o)))
    c = w.contracts[:n]
    assert np.array_equal(host(d_px, np.float64, (n,)), ope.batch_bates(c, w.params[0], tol=w.tol))
    assert host(d_gr, ope.RESULT_DTYPE, (n,)).tobytes() == ope.batch_bates_greeks(c, w.params[0], tol=w.tol).tobytes()
    assert host(d_ga, ope.RESULT_DTYPE, (n,)).tobytes() == \
        ope.batch_greeks_ad(ope.MODEL_BATES, c, w.params[0], tol=w.tol).tobytes()


def test_gradient_and_implied_vol(ope, env):
    torch, st, lib, opts, dev, host = env
    w = W.c2(n_surf=16, seed=43)
    o = opts(w.tol)
    d_con, d_off, d_par = dev(w.contracts), dev(w.surf_offsets), dev(w.params)
    d_p = torch.empty(w.n * 8, dtype=torch.uint8, device="cuda")
    d_g = torch.empty(w.n * 5 * 8, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(st):
        _ok(ope, lib.ope_price_gradient_surfaces(0, d_con.data_ptr(), w.n, d_off.data_ptr(), w.n_surf,
                                                 d_par.data_ptr(), d_p.data_ptr(), d_g.data_ptr(), ctypes.byref(o)))
    rp, rg = ope.price_gradient_surfaces(ope.MODEL_HESTON, w.contracts, w.surf_offsets, w.params, tol=w.tol)
    assert np.array_equal(host(d_p, np.float64, (w.n,)), rp)
    assert np.array_equal(host(d_g, np.float64, (w.n, 5)), rg)
    # implied vols of those prices
    d_iv = torch.empty(w.n * 8, dtype=torch.uint8, device="cuda")
    d_ok = torch.empty(w.n * 4, dtype=torch.uint8, device="cuda")
    d_px = dev(rp)
    with torch.cuda.stream(st):
        _ok(ope, lib.ope_batch_implied_vol(d_con.data_ptr(), w.n, d_px.data_ptr(), d_iv.data_ptr(), d_ok.data_ptr(),
                                           ctypes.byref(o)))
    iv, ok = ope.batch_implied_vol(w.contracts, rp)
    assert np.array_equal(host(d_iv, np.float64, (w.n,)), iv)
    assert np.array_equal(host(d_ok, np.int32, (w.n,)).astype(bool), np.asarray(ok).astype(bool))


def test_calibration(ope, env, oracle):
    torch, st, lib, opts, dev, host = env

    def price_fn(cc, params, sidx):
        off = np.concatenate([[0], np.cumsum(np.bincount(sidx, minlength=params.shape[0]))])
        return ope.price_surfaces(ope.MODEL_HESTON, cc, off, params, tol=1e-10)

    con, iv, off, tp, p0 = W.c4(price_fn, ope.batch_implied_vol, n_surf=3, seed=45)
    o = opts(1e-8)
    d_con, d_iv, d_off, d_p0 = dev(con), dev(iv), dev(off), dev(p0)
    d_out = torch.empty(3 * ope.CALIB_RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(st):
        _ok(ope, lib.ope_calibrate_surfaces(0, d_con.data_ptr(), d_iv.data_ptr(), None, con.size, d_off.data_ptr(), 3,
                                            d_p0.data_ptr(), d_out.data_ptr(), ctypes.byref(o)))
    got = host(d_out, ope.CALIB_RESULT_DTYPE, (3,))
    ref = ope.calibrate_surfaces(ope.MODEL_HESTON, con, iv, off, p0)
    assert got.tobytes() == ref.tobytes()


def test_calls_on_different_streams_are_ordered(ope, env):
    """A device-pointer call on one stream, then at once a host-pointer call
    (the library's own stream) and a device-pointer call on a second stream,
    all from this thread: they share the thread's workspace, so each later
    call must wait on the device for the earlier one's work."""
    torch, st, lib, opts, dev, host = env
    big = W.c3(n=65536, per_surface=256, seed=47)
    small = W.c3(n=4096, per_surface=256, seed=48)
    want_big = ope.price_surfaces(ope.MODEL_BATES, big.contracts, big.surf_offsets, big.params, tol=big.tol)
    want_small = ope.price_surfaces(ope.MODEL_BATES, small.contracts, small.surf_offsets, small.params, tol=small.tol)
    st2 = torch.cuda.Stream()
    o1 = opts(big.tol)
    o2 = ope._lib.Options(tol=small.tol, flags=ope._lib.FLAG_DEVICE_PTRS, reserved=0, stream=st2.cuda_stream)
    b = [dev(big.contracts), dev(big.surf_offsets), dev(big.params)]
    s = [dev(small.contracts), dev(small.surf_offsets), dev(small.params)]
    for _ in range(3):
        d_big = torch.full((big.n,), -1.0, dtype=torch.float64, device="cuda")
        d_small = torch.full((small.n,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        _ok(ope, lib.ope_price_surfaces(1, b[0].data_ptr(), big.n, b[1].data_ptr(), big.n_surf, b[2].data_ptr(),
                                        d_big.data_ptr(), ctypes.byref(o1)))
        got_host = ope.price_surfaces(ope.MODEL_BATES, small.contracts, small.surf_offsets, small.params,
                                      tol=small.tol)
        _ok(ope, lib.ope_price_surfaces(1, s[0].data_ptr(), small.n, s[1].data_ptr(), small.n_surf, s[2].data_ptr(),
                                        d_small.data_ptr(), ctypes.byref(o2)))
        torch.cuda.synchronize()
        assert np.array_equal(got_host, want_small)
        assert np.array_equal(d_big.cpu().numpy(), want_big)
        assert np.array_equal(d_small.cpu().numpy(), want_small)
