"""GPU: ope_price_surfaces_noalloc, the entry point for callers that cannot
let the library allocate device memory (pricing under stream capture, latency
paths that cannot take cudaMalloc/cudaFree's synchronisation, hosts whose
device memory belongs to another allocator).  Its scratch is a static device
array shared by every call, so this checks two calls in a row (the shared
counters must be cleared each time) against the allocating entry point, at
the price tolerance the other GPU tests use (1e-9 * S).  Collected last on
purpose: a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRICE_TOL = 1e-9 * 100.0


def _noalloc(L, model, d_con, n, d_off, n_surf, d_par, d_out, tol, stream):
    return L.ope_price_surfaces_noalloc(model, d_con.data_ptr(), n, d_off.data_ptr(), n_surf, d_par.data_ptr(),
                                        d_out.data_ptr(), tol, stream)


def test_noalloc_matches_allocating_entry_point_twice(ope):
    import torch

    from ope_b200 import _lib
    from ope_b200 import workloads as W

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream().cuda_stream
    for model, w in ((ope.MODEL_BATES, W.c3(n=1 << 14, per_surface=256)), (ope.MODEL_HESTON, W.c2(n_surf=40))):
        assert w.n <= 65536
        ref = ope.price_surfaces(model, w.contracts, w.surf_offsets, w.params, tol=w.tol)
        d_con = torch.from_numpy(w.contracts.view(np.uint8).copy()).to(dev)
        d_off = torch.from_numpy(w.surf_offsets.copy()).to(dev)
        d_par = torch.from_numpy(w.params.copy()).to(dev)
        for _ in range(2):
            d_out = torch.full((w.n,), float("nan"), dtype=torch.float64, device=dev)
            _lib.check(_noalloc(L, model, d_con, w.n, d_off, w.n_surf, d_par, d_out, w.tol, stream))
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert float(np.max(np.abs(got - ref))) <= PRICE_TOL


def test_noalloc_rejects_oversized_calls(ope):
    from ope_b200 import _lib

    L = _lib.load()
    rc = L.ope_price_surfaces_noalloc(ope.MODEL_HESTON, 1, 65537, 1, 1, 1, 1, 1e-8, None)
    assert rc == 1  # OPE_ERR_INVALID_ARG before any device access
    assert b"OPE_NOALLOC_MAX_CONTRACTS" in L.ope_last_error()
