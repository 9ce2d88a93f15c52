"""GPU: the request server (continuous batching, admission by device memory).

The serving contract: a request's results are the same (bit for bit) whether
it runs alone or mixed with others, and equal the direct API's; requests that
can never fit the admission budget are rejected; pending requests can be
cancelled; a NaN request poisons only itself.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _submit(srv, r):
    from ope_b200 import MODEL_BATES, MODEL_HESTON

    if r.kind == 0:
        return srv.submit_price(MODEL_BATES, r.contracts, r.params)
    return srv.submit_calibrate(MODEL_HESTON, r.contracts, r.iv, r.params)


def _same(a, b):
    return np.asarray(a).tobytes() == np.asarray(b).tobytes()


def test_alone_equals_in_mix_and_direct_api(ope):
    from ope_b200 import serving as SV

    reqs = SV.make_stream(30, seed=3)
    assert any(r.kind == 1 for r in reqs) and any(r.kind == 0 for r in reqs)
    nan_req = SV.StreamRequest(0, reqs[0].contracts.copy(), reqs[0].params.copy())
    nan_req.params[1] = np.nan
    mix = reqs[:15] + [nan_req] + reqs[15:]
    with SV.Server(hbm_cap_bytes=2 << 30, max_inflight=4) as srv:
        ids = [_submit(srv, r) for r in mix]
        mixed = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
        alone = [srv.wait(_submit(srv, r))[0] for r in mix]
    assert st["completed"] == len(mix) and st["batches"] < len(mix)  # batched
    for k, (a, b) in enumerate(zip(mixed, alone)):
        assert _same(a, b), k
    # reprices equal the direct batch API; calibrations equal the direct LM API
    for r, got in zip(mix, mixed):
        if r.kind == 0:
            assert _same(got, ope.batch_bates(r.contracts, r.params))
        else:
            direct = ope.calibrate_surfaces(ope.MODEL_HESTON, r.contracts, r.iv, [0, r.contracts.size],
                                            r.params[None])[0]
            assert _same(got, direct)


def test_overlapping_batches(ope):
    from ope_b200 import serving as SV

    reqs = [r for r in SV.make_stream(60, seed=11) if r.kind == 0]
    with SV.Server(hbm_cap_bytes=2 << 30, max_inflight=4, max_batch_contracts=4000) as srv:
        ids = [_submit(srv, r) for r in reqs]
        for i in ids:
            srv.wait(i)
        st = srv.stats()
    assert st["max_inflight"] >= 2, st


def test_admission_rejects_oversized_request(ope):
    from ope_b200 import serving as SV
    from ope_b200 import workloads as W

    w = W.c3(n=1 << 16, per_surface=1 << 16)
    small = w.contracts[:100]
    with SV.Server(hbm_cap_bytes=4 << 20) as srv:  # 4 MiB budget
        big = srv.submit_price(ope.MODEL_BATES, w.contracts, w.params[0])
        ok = srv.submit_price(ope.MODEL_BATES, small, w.params[0])
        with pytest.raises(ope.OpeError) as e:
            srv.wait(big)
        assert e.value.status == SV.OPE_ERR_REJECTED
        px, _ = srv.wait(ok)
        assert _same(px, ope.batch_bates(small, w.params[0]))
        assert srv.stats()["rejected"] == 1


def test_cancel_and_timeout(ope):
    from ope_b200 import serving as SV
    from ope_b200 import workloads as W

    w = W.c3(n=1 << 18, per_surface=1 << 18)
    with SV.Server(hbm_cap_bytes=1 << 30, max_inflight=1) as srv:
        long_id = srv.submit_price(ope.MODEL_BATES, w.contracts, w.params[0])  # occupies the only slot
        queued = srv.submit_price(ope.MODEL_BATES, w.contracts[:50], w.params[0])
        srv.cancel(queued)
        with pytest.raises(ope.OpeError) as e:
            srv.wait(queued)
        assert e.value.status == SV.OPE_ERR_CANCELLED
        with pytest.raises(ope.OpeError) as e:
            srv.wait(long_id, timeout_ms=0.0)
        assert e.value.status == SV.OPE_ERR_TIMEOUT
        px, ms = srv.wait(long_id)
        assert np.all(np.isfinite(px)) and ms > 0


def test_batch_implied_vol_matches_oracle(ope, oracle):  # batch.rs:51-56, 255-264; iv.rs:97-129
    rng = np.random.default_rng(4)
    n = 4000
    con = oracle.contracts(100.0, 100.0 * np.exp(rng.uniform(-0.5, 0.5, n)), np.exp(rng.uniform(np.log(0.02), 0.0, n)),
                           rng.uniform(0.0, 0.06, n), rng.uniform(0.0, 0.03, n), rng.integers(0, 2, n),
                           vol=rng.uniform(0.05, 1.0, n))
    px = np.array([oracle.bsm_price(c) for c in con])
    px[:10] = -1.0  # rejected by the bounds check (iv.rs:23)
    iv, ok = ope.batch_implied_vol(con, px)
    ref, rok = oracle.batch_implied_vol(con, px)
    assert not ok[:10].any()
    # where the time value is below 1e-9 * S the price equals intrinsic to the last ulps, the
    # IV is not identifiable in double precision and the bounds check (iv.rs:30) flips with the
    # last ulp of exp(); everywhere else the two solvers must agree on success and value
    eq, er = np.exp(-con["div_yield"] * con["expiry"]), np.exp(-con["rate"] * con["expiry"])
    intr = np.where(con["opt_type"] == 0, np.maximum(con["spot"] * eq - con["strike"] * er, 0.0),
                    np.maximum(con["strike"] * er - con["spot"] * eq, 0.0))
    well = (px - intr) > 1e-9 * 100.0
    assert well.sum() > 3000
    assert np.array_equal(ok[well], rok[well])
    both = well & ok & rok
    # both solvers stop once |price error| < 1e-10 (iv.rs:69), so each IV is known to 1e-10 / vega
    vt = ref * np.sqrt(con["expiry"])
    d1 = (np.log(con["spot"] / con["strike"]) + (con["rate"] - con["div_yield"] + 0.5 * ref * ref) * con["expiry"]) / vt
    vega = con["spot"] * eq * np.exp(-0.5 * d1 * d1) / np.sqrt(2 * np.pi) * np.sqrt(con["expiry"])
    lim = 2.5e-10 / np.maximum(vega, 1e-300) + 1e-12
    assert np.all(np.abs(iv[both] - ref[both]) <= lim[both])
    good = both & (px > 1e-6)
    assert np.max(np.abs(iv[good] - con["vol"][good])) < 1e-6
