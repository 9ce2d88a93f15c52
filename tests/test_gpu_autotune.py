"""GPU: the launch-shape autotuner of the pricing kernel (ope_autotune).  It
measures every candidate shape -- warps per block, deepest-first or input
order, full or half occupancy -- per size class on this device and installs
a table; every shape must give the same prices bit for bit (a unit's
arithmetic does not depend on scheduling), so tuned and untuned calls of
every size class are compared here, along with the oracle on a sample."""
import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_tuned_table_is_sane(ope):
    rows = ope.autotune(ope.MODEL_BATES, quick=True)
    assert len(rows) == 16 and rows[-1]["max_contracts"] is None
    assert [r["max_contracts"] for r in rows[:-1]] == [1 << k for k in range(6, 21)]
    for r in rows[:12]:  # the classes a quick tuning measures (up to 2^17 contracts)
        assert r["warps_per_block"] in (1, 2, 4) and 0.0 < r["occupancy"] <= 1.0
        assert 0.0 < r["ms_tuned"] <= r["ms_default"]
        if (r["warps_per_block"], r["deepest_first"], r["occupancy"]) != (4, False, 1.0):
            assert r["ms_tuned"] < 0.97 * r["ms_default"]  # kept only when it beats the default by 3 %
    table, tuned = ope.tune_table(ope.MODEL_BATES)
    assert tuned and table == rows
    print("\n".join(str(r) for r in rows))


@pytest.mark.parametrize("model", ["heston", "bates"])
def test_tuned_and_default_shapes_price_identically(ope, oracle, model):
    m = ope.MODEL_BATES if model == "bates" else ope.MODEL_HESTON
    ope.autotune(m, quick=True)
    w = W.c3(n=1 << 15, per_surface=256, seed=61) if model == "bates" else W.c2(n_surf=160, seed=61)
    for n_surf in (1, 4, 16, w.n_surf):  # 256 .. all contracts: several size classes
        sub = w.subset(list(range(min(n_surf, w.n_surf))))
        ope.set_autotune(True)
        tuned = ope.price_surfaces(m, sub.contracts, sub.surf_offsets, sub.params, tol=sub.tol)
        ope.set_autotune(False)
        plain = ope.price_surfaces(m, sub.contracts, sub.surf_offsets, sub.params, tol=sub.tol)
        ope.set_autotune(True)
        assert np.array_equal(tuned, plain)
    # the plain per-surface drop-in too, and the oracle on a sample
    one = w.subset([0])
    got = (ope.batch_bates if model == "bates" else ope.batch_heston)(one.contracts, one.params[0], tol=one.tol)
    ref = oracle.batch_price(one.contracts, one.params, model == "bates", one.tol)
    assert float(np.max(np.abs(got - ref))) <= 1e-9 * 100.0


def test_every_shape_prices_identically(ope):
    """Each of the twelve shapes the tuner chooses from, installed as the
    table of every class (ope_set_tune_table): a 3,000-contract multi-surface
    call and a 64-contract one price exactly as the default shape does."""
    w = W.c3(n=3072, per_surface=256, seed=67)
    small = w.subset([0])
    small.contracts, small.surf_offsets = small.contracts[:64], np.array([0, 64], np.int64)
    ope.set_autotune(False)
    ref = ope.price_surfaces(ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, tol=w.tol)
    ref_small = ope.price_surfaces(ope.MODEL_BATES, small.contracts, small.surf_offsets, small.params, tol=w.tol)
    ope.set_autotune(True)
    saved, _ = ope.tune_table(ope.MODEL_BATES)
    try:
        for warps in (1, 2, 4):
            for deepest in (False, True):
                for occ in (1.0, 0.5):
                    rows = [dict(r, warps_per_block=warps, deepest_first=deepest, occupancy=occ) for r in saved]
                    ope.set_tune_table(ope.MODEL_BATES, rows)
                    assert ope.tune_table(ope.MODEL_BATES)[0][3]["warps_per_block"] == warps
                    got = ope.price_surfaces(ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, tol=w.tol)
                    assert np.array_equal(got, ref), (warps, deepest, occ)
                    got = ope.price_surfaces(ope.MODEL_BATES, small.contracts, small.surf_offsets, small.params,
                                             tol=w.tol)
                    assert np.array_equal(got, ref_small), (warps, deepest, occ)
    finally:
        ope.set_tune_table(ope.MODEL_BATES, saved)
    with pytest.raises(ope.OpeError):
        ope.set_tune_table(ope.MODEL_BATES, [dict(r, warps_per_block=3) for r in saved])
