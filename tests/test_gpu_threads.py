"""GPU: concurrent host threads (the ABI is thread-safe; each thread owns its
stream and workspace).  Eight threads price, differentiate and calibrate at
the same time; every result equals the same call made alone."""
import threading

import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_concurrent_threads_equal_serial(ope):
    w = W.c3(n=8 * 2048, per_surface=256, seed=51)
    parts = [w.subset(list(range(8 * k, 8 * k + 8))) for k in range(8)]
    serial = [ope.price_surfaces(ope.MODEL_BATES, p.contracts, p.surf_offsets, p.params, tol=p.tol) for p in parts]
    sgrad = [ope.price_gradient_surfaces(ope.MODEL_BATES, p.contracts[:512], p.surf_offsets[:3], p.params[:2],
                                         tol=p.tol)[1] for p in parts]
    results, grads, errors = [None] * 8, [None] * 8, []

    def work(k):
        try:
            p = parts[k]
            for _ in range(3):
                results[k] = ope.price_surfaces(ope.MODEL_BATES, p.contracts, p.surf_offsets, p.params, tol=p.tol)
                grads[k] = ope.price_gradient_surfaces(ope.MODEL_BATES, p.contracts[:512], p.surf_offsets[:3],
                                                       p.params[:2], tol=p.tol)[1]
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(repr(e))

    threads = [threading.Thread(target=work, args=(k,)) for k in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for k in range(8):
        assert np.array_equal(results[k], serial[k])
        assert np.array_equal(grads[k], sgrad[k])


def test_workspace_growth_does_not_drain_other_streams(ope):
    """A thread whose workspace grows (its first call, then a larger one) must
    not wait for, or stall, work another thread has queued on its own stream:
    growth is stream-ordered (cudaFreeAsync / cudaMallocAsync), with no device
    synchronisation.  Thread A queues ten launches of a 512k-contract Bates
    batch (about 25 ms each) on its stream; thread B then makes two growing
    host-pointer calls.  B's calls must return while A's stream is still busy,
    with B's prices equal to the same calls made alone."""
    import torch

    dev = torch.device("cuda", 0)
    w = W.c3(n=1 << 19, per_surface=256, seed=53)
    small = [w.subset([0]), w.subset(list(range(1, 17)))]
    alone = [ope.price_surfaces(ope.MODEL_BATES, p.contracts, p.surf_offsets, p.params, tol=p.tol) for p in small]
    d_con = torch.from_numpy(w.contracts.view(np.uint8).copy()).to(dev)
    d_off = torch.from_numpy(w.surf_offsets.copy()).to(dev)
    d_par = torch.from_numpy(w.params.copy()).to(dev)
    d_out = torch.empty(w.n, dtype=torch.float64, device=dev)
    sa = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    got, errors = [None, None], []

    def thread_b():
        try:
            for k, p in enumerate(small):
                got[k] = ope.price_surfaces(ope.MODEL_BATES, p.contracts, p.surf_offsets, p.params, tol=p.tol)
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(repr(e))

    for _ in range(10):
        ope.price_surfaces_device(ope.MODEL_BATES, d_con, w.n, d_off, w.n_surf, d_par, d_out, tol=w.tol,
                                  stream=sa.cuda_stream)
    b = threading.Thread(target=thread_b)
    b.start()
    b.join(timeout=120)
    a_busy = not sa.query()
    sa.synchronize()
    assert not errors, errors
    assert a_busy, "thread B's calls returned only after thread A's stream had drained"
    for k in range(2):
        assert np.array_equal(got[k], alone[k])
