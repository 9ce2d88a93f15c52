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
