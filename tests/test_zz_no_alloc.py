"""GPU: ope_price_surfaces_noalloc, the entry point for callers that cannot
let the library allocate device memory -- a host that hands all of a GPU's
memory to one allocator (a framework's caching allocator, or a fixed arena
sized at start-up) has none left for a library's own cudaMalloc, and a
latency-critical request path cannot afford cudaMalloc/cudaFree, either of
which may wait for the whole device.

Its scratch is a static device array shared by every call, so this checks two
calls in a row (the shared counters must be cleared each time) against the
allocating entry point and against the oracle, at the price tolerance the
other GPU tests use (1e-9 * S), including a call at the size limit; and that
a call allocates nothing: a fresh host thread that only calls this entry point
has no library workspace afterwards, and the device's free memory is the same
before and after a call.  Collected last on purpose: a failure here leaves
every other test already run.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

S = 100.0
PRICE_TOL = 1e-9 * S
MAX_N = 65536  # OPE_NOALLOC_MAX_CONTRACTS


def _noalloc(L, model, d_con, n, d_off, n_surf, d_par, d_out, tol, stream):
    return L.ope_price_surfaces_noalloc(model, d_con.data_ptr(), n, d_off.data_ptr(), n_surf, d_par.data_ptr(),
                                        d_out.data_ptr(), tol, stream)


def _device_inputs(w, dev):
    import torch

    return (torch.from_numpy(w.contracts.view(np.uint8).copy()).to(dev),
            torch.from_numpy(w.surf_offsets.copy()).to(dev),
            torch.from_numpy(w.params.copy()).to(dev))


def test_noalloc_matches_allocating_entry_point_and_oracle_twice(ope, oracle):
    import torch

    from ope_b200 import _lib
    from ope_b200 import workloads as W

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream().cuda_stream
    # the Bates call is exactly at the size limit
    for model, w in ((ope.MODEL_BATES, W.c3(n=MAX_N, per_surface=256)), (ope.MODEL_HESTON, W.c2(n_surf=40))):
        assert w.n <= MAX_N
        ref = ope.price_surfaces(model, w.contracts, w.surf_offsets, w.params, tol=w.tol)
        rng = np.random.default_rng(11)
        pick = np.sort(rng.choice(w.n, min(w.n, 1500), replace=False))
        orc = oracle.batch_price(w.contracts[pick], w.params, model == ope.MODEL_BATES, w.tol,
                                 surf_idx=w.surf_idx()[pick])
        d_con, d_off, d_par = _device_inputs(w, dev)
        for _ in range(2):
            d_out = torch.full((w.n,), float("nan"), dtype=torch.float64, device=dev)
            _lib.check(_noalloc(L, model, d_con, w.n, d_off, w.n_surf, d_par, d_out, w.tol, stream))
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert float(np.max(np.abs(got - ref))) <= PRICE_TOL
            assert float(np.max(np.abs(got[pick] - orc))) <= PRICE_TOL


def test_noalloc_allocates_nothing(ope):
    """A fresh host thread that calls only this entry point ends with no
    library workspace, and the device's free memory does not move across its
    calls (measured after the first call on the device, which does the
    one-time set-up)."""
    import torch

    from ope_b200 import _lib
    from ope_b200 import workloads as W

    L = _lib.load()
    dev = torch.device("cuda", 0)
    w = W.c3(n=4096, per_surface=256)
    d_con, d_off, d_par = _device_inputs(w, dev)
    outs = [torch.empty(w.n, dtype=torch.float64, device=dev) for _ in range(3)]
    torch.cuda.synchronize()
    seen = {}

    def worker():
        torch.cuda.set_device(dev)
        s = torch.cuda.Stream(device=dev)
        st = s.cuda_stream
        _lib.check(_noalloc(L, ope.MODEL_BATES, d_con, w.n, d_off, w.n_surf, d_par, outs[0], w.tol, st))
        s.synchronize()
        free0, _ = torch.cuda.mem_get_info(dev)
        alloc0 = torch.cuda.memory_allocated(dev)
        for o in outs[1:]:
            _lib.check(_noalloc(L, ope.MODEL_BATES, d_con, w.n, d_off, w.n_surf, d_par, o, w.tol, st))
        s.synchronize()
        seen["free"] = (free0, torch.cuda.mem_get_info(dev)[0])
        seen["alloc"] = (alloc0, torch.cuda.memory_allocated(dev))
        seen["workspace"] = int(L.ope_workspace_bytes())

    t = threading.Thread(target=worker)
    t.start()
    t.join()
    assert seen["workspace"] == 0
    assert seen["free"][0] == seen["free"][1], seen["free"]
    assert seen["alloc"][0] == seen["alloc"][1]
    ref = ope.price_surfaces(ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, tol=w.tol)
    for o in outs:
        assert float(np.max(np.abs(o.cpu().numpy() - ref))) <= PRICE_TOL


def test_noalloc_rejects_oversized_calls_and_bad_tolerances(ope):
    from ope_b200 import _lib

    L = _lib.load()
    rc = L.ope_price_surfaces_noalloc(ope.MODEL_HESTON, 1, MAX_N + 1, 1, 1, 1, 1, 1e-8, None)
    assert rc == 1  # OPE_ERR_INVALID_ARG before any device access
    assert b"OPE_NOALLOC_MAX_CONTRACTS" in L.ope_last_error()
    for tol in (float("inf"), float("nan")):
        assert L.ope_price_surfaces_noalloc(ope.MODEL_HESTON, 1, 16, 1, 1, 1, 1, tol, None) == 1
        assert b"tol" in L.ope_last_error()
