"""GPU: the run kernel (k_price_runs) -- consecutive contracts of one surface
with the same expiry and rate share the characteristic function's values
at every panel they both bisect (the run cache), and only the phase
u ln(S/K) is per strike.  The cache holds exactly what the per-contract
evaluation computes, so every mode must give bit-identical prices: one
contract per unit, the automatic mode (a device probe of the runs), and
fixed blocks of 2..32 contracts -- on grid surfaces laid out expiry by
expiry, on layouts without runs, with runs straddling block boundaries,
with a run too deep for the cache, and with NaN parameters.  Prices are
checked against the oracle (heston.rs / bates.rs restated) on a sample at
the price tolerance of the other GPU tests (1e-9 * S)."""
import numpy as np
import pytest

from ope_b200 import workloads as W

pytestmark = pytest.mark.gpu

S = 100.0
PRICE_TOL = 1e-9 * S
MODES = (1, 0, 2, 8, 16, 32)  # per_unit: one, automatic, fixed blocks


@pytest.fixture
def per_unit(ope):
    """Sets every size class of a model's launch table to one contracts-per-unit
    mode; restores the table (as the default entries when it was untuned)."""
    saved = {m: ope.tune_table(m)[0] for m in (ope.MODEL_HESTON, ope.MODEL_BATES)}

    def set_mode(model, pu):
        rows = [dict(r) for r in saved[model]]
        for r in rows:
            r.update(warps_per_block=4, deepest_first=False, occupancy=1.0, per_unit=pu)
        ope.set_tune_table(model, rows)

    yield set_mode
    for m, rows in saved.items():
        ope.set_tune_table(m, rows)


def _bates_params(p5, seed):
    r = np.random.default_rng(seed)
    ns = p5.shape[0]
    return np.concatenate([p5, r.uniform(0, 1.5, (ns, 1)), r.uniform(-0.3, 0.1, (ns, 1)),
                           r.uniform(0.05, 0.4, (ns, 1))], axis=1)


def _grid(n_surf, seed=21, strike_major_every=0, bates=False):
    """c2-like surfaces (uneven strike x expiry grids, expiry-major, so each
    expiry's strikes are one run); every strike_major_every-th surface is laid
    out strike by strike instead (runs of one contract)."""
    w = W.c2(n_surf=n_surf, seed=seed)
    con, off = w.contracts.copy(), w.surf_offsets
    if strike_major_every:
        for s in range(0, n_surf, strike_major_every):
            a, b = off[s], off[s + 1]
            blk = con[a:b]
            con[a:b] = blk[np.lexsort((blk["expiry"], blk["strike"]))]
    params = _bates_params(w.params, seed) if bates else w.params
    return con, off, params


def _prices(ope, model, con, off, params):
    return ope.price_surfaces(model, con, off, params, tol=1e-10)


def _all_modes(ope, per_unit, model, con, off, params, modes=MODES):
    """Prices in each mode through device buffers, every call into an output
    filled with NaN (a launch that did no work cannot pass for one that did),
    and the contracts per unit each call used."""
    import torch

    dev = torch.device("cuda", 0)
    d_con = torch.from_numpy(con.view(np.uint8).copy()).to(dev)
    d_off = torch.from_numpy(off.copy()).to(dev)
    d_par = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float64)).to(dev)
    out, used = {}, {}
    for pu in modes:
        per_unit(model, pu)
        d_out = torch.full((con.size,), float("nan"), dtype=torch.float64, device=dev)
        ope.price_surfaces_device(model, d_con, con.size, d_off, off.size - 1, d_par, d_out, tol=1e-10)
        used[pu] = ope.last_per_unit()
        out[pu] = d_out.cpu().numpy()
    for pu in modes:
        if pu >= 1:
            assert used[pu] == pu, (pu, used[pu])
    return out, used


def _assert_bitwise(out):
    ref = out[1].view(np.int64)
    for pu, got in out.items():
        assert np.array_equal(got.view(np.int64), ref), (pu, float(np.nanmax(np.abs(got - out[1]))))


@pytest.mark.parametrize("bates", [False, True])
def test_grid_surfaces_bitwise_in_every_mode_and_match_oracle(ope, oracle, per_unit, bates):
    model = ope.MODEL_BATES if bates else ope.MODEL_HESTON
    con, off, params = _grid(160 if bates else 220, bates=bates)
    assert con.size >= 32768  # the automatic mode probes calls of this size
    out, _ = _all_modes(ope, per_unit, model, con, off, params)
    _assert_bitwise(out)
    rng = np.random.default_rng(5)
    pick = np.sort(rng.choice(con.size, 600, replace=False))
    sidx = np.repeat(np.arange(off.size - 1), np.diff(off))
    orc = oracle.batch_price(con[pick], params, bates, 1e-10, surf_idx=sidx[pick])
    assert float(np.max(np.abs(out[0][pick] - orc))) <= PRICE_TOL


def test_layouts_without_runs_and_runs_across_blocks(ope, per_unit):
    """Strike-major surfaces (runs of one), expiry-major ones, one-contract
    surfaces, and a rate change inside an expiry: every split of the runs by
    the blocks gives the same bits."""
    con, off, params = _grid(200, seed=22, strike_major_every=3)
    # one-contract surfaces at the front, and a rate change halfway through
    # each expiry of surface 5 (same expiry, different rate: two runs)
    a, b = off[5], off[6]
    con[a:b]["rate"][::2] += 1e-3
    singles = con[:7].copy()
    con = np.concatenate([singles, con])
    off = np.concatenate([np.arange(8, dtype=np.int64), off[1:] + 7])
    params = np.concatenate([params[:7], params])
    _assert_bitwise(_all_modes(ope, per_unit, ope.MODEL_HESTON, con, off, params)[0])


def test_scattered_expiries_auto_mode_matches_per_contract(ope, per_unit):
    """No two contracts share an expiry (the deep-wing Bates batch): the probe
    keeps the per-contract kernel, and every mode gives the same bits."""
    w = W.c3(n=40000, per_surface=256)
    out, used = _all_modes(ope, per_unit, ope.MODEL_BATES, w.contracts, w.surf_offsets, w.params, modes=(1, 0, 16))
    _assert_bitwise(out)
    assert used[0] == 1


def test_auto_mode_takes_the_run_kernel_on_a_large_grid(ope, oracle, per_unit):
    """About 320k grid contracts: the probe picks blocks of 4 or more contracts,
    and the prices equal one-contract-per-unit prices bit for bit."""
    con, off, params = _grid(900, seed=25)
    out, used = _all_modes(ope, per_unit, ope.MODEL_HESTON, con, off, params, modes=(1, 0))
    assert used[0] >= 4, used
    _assert_bitwise(out)
    pick = np.sort(np.random.default_rng(6).choice(con.size, 400, replace=False))
    sidx = np.repeat(np.arange(off.size - 1), np.diff(off))
    orc = oracle.batch_price(con[pick], params, False, 1e-10, surf_idx=sidx[pick])
    assert float(np.max(np.abs(out[0][pick] - orc))) <= PRICE_TOL


def test_run_deeper_than_the_cache_and_nan_parameters(ope, per_unit):
    """A run of short-dated deep-wing strikes (integrals of up to 200 panels:
    more panels than the 128-entry cache holds, so later ones are evaluated
    uncached) and a surface with NaN parameters."""
    m = np.linspace(-1.2, 0.7, 40)
    rows = []
    for t in (1.0 / 365, 2.0 / 365, 0.05):
        for x in m:
            rows.append((S, S * np.exp(x), t, 0.02, 0.01, 0.2, int(x > 0), 0))
    deep = np.array(rows, dtype=W.CONTRACT_DTYPE)
    con, off, params = _grid(150, seed=23)
    con = np.concatenate([deep, deep, con])
    off = np.concatenate([[0, deep.size, 2 * deep.size], off[1:] + 2 * deep.size]).astype(np.int64)
    p_deep = np.array([[0.04, 1.5, 0.04, 0.9, -0.9], [np.nan, 1.5, 0.04, 0.5, -0.7]])
    params = np.concatenate([p_deep, params])
    _assert_bitwise(_all_modes(ope, per_unit, ope.MODEL_HESTON, con, off, params)[0])
    # one integral of 64 bisections evaluates 129 panels: more than the cache holds
    nb = np.zeros(2 * deep.size, np.int32)
    ope.price_surfaces(ope.MODEL_HESTON, deep, np.array([0, deep.size], np.int64), params[:1], tol=1e-10,
                       bisections=nb)
    assert int(nb.max()) >= 64


def test_host_paths_agree_with_device_pointers(ope, per_unit):
    """Pageable host buffers (copied, in two overlapped parts from 262,144
    contracts), pinned ones (used in place) and device buffers, with the run
    kernel in a fixed mode: the same bits."""
    import torch

    con, off, params = _grid(800, seed=24)
    assert con.size >= 262144
    dev_out, _ = _all_modes(ope, per_unit, ope.MODEL_HESTON, con, off, params, modes=(8,))
    per_unit(ope.MODEL_HESTON, 8)
    pageable = _prices(ope, ope.MODEL_HESTON, con, off, params)
    pinned_in = torch.from_numpy(con.view(np.uint8).copy()).pin_memory()
    pinned_out = torch.full((con.size,), float("nan"), dtype=torch.float64).pin_memory()
    ope.price_surfaces(ope.MODEL_HESTON, pinned_in.numpy().view(W.CONTRACT_DTYPE), off, params, tol=1e-10,
                       out=pinned_out.numpy())
    for got in (pageable, pinned_out.numpy()):
        assert np.array_equal(got.view(np.int64), dev_out[8].view(np.int64))


def test_tune_table_rejects_bad_per_unit(ope):
    rows, _ = ope.tune_table(ope.MODEL_HESTON)
    bad = [dict(r, per_unit=33) for r in rows]
    with pytest.raises(Exception, match="per_unit"):
        ope.set_tune_table(ope.MODEL_HESTON, bad)


def test_workspace_limit_drops_the_run_cache_not_the_call(ope, per_unit):
    """Under a workspace limit too small for the run cache (~157 MB) but large
    enough for the call itself, an automatic grid call still prices: it takes
    one contract per unit, with the same bits as the run kernel."""
    con, off, params = _grid(900, seed=26)
    per_unit(ope.MODEL_HESTON, 0)
    ref = _prices(ope, ope.MODEL_HESTON, con, off, params)
    chosen = ope.last_per_unit()
    assert chosen >= 4
    try:
        ope.set_workspace_limit(96 << 20)  # releases the workspace the probe's word was in
        assert ope.last_per_unit() == chosen
        got = _prices(ope, ope.MODEL_HESTON, con, off, params)
        assert ope.last_per_unit() == 1
    finally:
        ope.set_workspace_limit(0)
    assert np.array_equal(got.view(np.int64), ref.view(np.int64))


def _wide_grid(rng, n_surf, bates):
    """Grid surfaces (expiry-major) over the wide ranges of the fuzz test:
    vol-of-vol up to 3, correlation up to +-0.99, mean reversion 0.05 to 20,
    expiries from one day to ten years, strikes deep in and out of the money,
    jump intensities up to 5."""
    parts, off, pars = [], [0], []
    for _ in range(n_surf):
        r, q = rng.uniform(-0.01, 0.08), rng.uniform(0.0, 0.05)
        ts = np.sort(np.exp(rng.uniform(np.log(1 / 365), np.log(10.0), rng.integers(2, 8))))
        ms = np.sort(rng.uniform(-2.0, 1.2, rng.integers(4, 24)))
        T, M = np.meshgrid(ts, ms, indexing="ij")
        c = np.zeros(T.size, W.CONTRACT_DTYPE)
        c["spot"], c["expiry"] = S, T.ravel()
        c["strike"] = S * np.exp((r - q) * T.ravel() + M.ravel() * np.sqrt(np.minimum(T.ravel(), 1.0)))
        c["rate"], c["div_yield"], c["vol"] = r, q, 0.2
        c["opt_type"] = rng.integers(0, 2, T.size)
        parts.append(c)
        off.append(off[-1] + c.size)
        p = [rng.uniform(0.005, 0.6), np.exp(rng.uniform(np.log(0.05), np.log(20.0))), rng.uniform(0.005, 0.6),
             rng.uniform(0.05, 3.0), rng.uniform(-0.99, 0.99)]
        if bates:
            p += [rng.uniform(0.0, 5.0), rng.uniform(-0.5, 0.3), rng.uniform(0.02, 0.6)]
        pars.append(p)
    return np.concatenate(parts), np.array(off, np.int64), np.array(pars)


@pytest.mark.parametrize("bates", [False, True])
def test_wide_range_grids_bitwise_in_the_run_kernel(ope, oracle, per_unit, bates):
    """Wide-range grids: the run kernel (8 contracts per unit) gives the
    per-contract kernel's bits, and both the oracle's prices to 1e-9 S on a
    sample (non-finite where the reference's formula is)."""
    rng = np.random.default_rng(4040 + bates)
    con, off, params = _wide_grid(rng, 700, bates)
    model = ope.MODEL_BATES if bates else ope.MODEL_HESTON
    out, used = _all_modes(ope, per_unit, model, con, off, params, modes=(1, 8))
    assert used[8] == 8
    a, b = out[1], out[8]
    assert np.array_equal(a.view(np.int64), b.view(np.int64))
    pick = np.sort(rng.choice(con.size, 800, replace=False))
    sidx = np.repeat(np.arange(off.size - 1), np.diff(off)).astype(np.int32)
    ref = oracle.batch_price(con[pick], params, bates, 1e-10, surf_idx=sidx[pick])
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(b[pick]), fin)
    assert float(np.max(np.abs(b[pick][fin] - ref[fin]))) <= PRICE_TOL
