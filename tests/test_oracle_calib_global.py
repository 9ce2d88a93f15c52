"""CPU: pin the oracle's multistart / differential-evolution / Tikhonov
calibration (calibration.rs:204-427) and its rand 0.8 restatement.

rand is not pinned by the reference's lock file, so the generator is pinned
two ways: (a) xoshiro256++ outputs derived by hand from its definition and a
pure-Python restatement of rand 0.8's seeding and samplers, written here
independently of the C++ one; (b) the numbers the reference's own calibration
tests record from their measured runs (calibration.rs:870-1234): the DE Bates
landing point "v0=1.64 vs true 0.04, kappa=21 vs true 2", the condition
numbers "~3.2e6" (Heston, good p0) and "~3.7e7" (Bates, good p0), the
regularised cost "0.0006 vol points", and the asserts of every multistart,
pruning, DE and regularisation test.  (b) only holds under rand 0.8's
SmallRng::seed_from_u64 (PCG32 seeding): with xoshiro's own SplitMix64
seeding no restart of multistart_beats_bad_single_start converges.
"""
import math

import numpy as np
import pytest

M64 = (1 << 64) - 1


# ---- an independent pure-Python restatement of rand 0.8 SmallRng ---------
def _rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & M64


class PyRng:
    def __init__(self, state4):
        self.s = list(state4)

    @classmethod
    def seed_from_u64(cls, state):  # rand_core 0.6 default seed_from_u64 (PCG32)
        words = []
        for _ in range(8):
            state = (state * 6364136223846793005 + 11634580027462260723) & M64
            xorshifted = (((state >> 18) ^ state) >> 27) & 0xFFFFFFFF
            rot = state >> 59
            words.append(((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & 0xFFFFFFFF)
        return cls([words[2 * k] | (words[2 * k + 1] << 32) for k in range(4)])

    def next_u64(self):
        s = self.s
        out = (_rotl((s[0] + s[3]) & M64, 23) + s[0]) & M64
        t = (s[1] << 17) & M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = _rotl(s[3], 45)
        return out

    def gen_range_f64(self, lo, hi):
        import struct
        while True:
            bits = (self.next_u64() >> 12) | 0x3FF0000000000000
            v = struct.unpack("<d", struct.pack("<Q", bits))[0]
            res = (v - 1.0) * (hi - lo) + lo
            if res < hi:
                return res

    def gen_range_usize(self, lo, hi):
        rng = hi - lo
        zone = ((rng << (64 - rng.bit_length())) & M64) - 1
        while True:
            m = self.next_u64() * rng
            if (m & M64) <= zone:
                return lo + (m >> 64)


def _splitmix64(x):  # mc.rs:337-343
    x = (x + 0x9E3779B97F4A7C15) & M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def test_xoshiro_known_answers(oracle):
    # From the definition with state (1, 2, 3, 4): rotl(1 + 4, 23) + 1 = 41943041,
    # then one state update gives rotl(7 + 6 * 2^45, 23) + 7 = 58720359.
    got = oracle.xoshiro_from_state([1, 2, 3, 4], 6)
    assert int(got[0]) == 41943041 and int(got[1]) == 58720359
    ref = PyRng([1, 2, 3, 4])
    assert [int(x) for x in got] == [ref.next_u64() for _ in range(6)]


def test_seeding_and_samplers_match_python_restatement(oracle):
    for seed in (0, 1, 777, 12345, 2**63 + 5, M64):
        assert oracle.splitmix64(seed) == _splitmix64(seed)
        r = PyRng.seed_from_u64(seed)
        assert [int(x) for x in oracle.small_rng_u64(seed, 8)] == [r.next_u64() for _ in range(8)]
        r = PyRng.seed_from_u64(seed)
        assert list(oracle.rng_gen_range_f64(seed, 0.02, 0.4, 16)) == [r.gen_range_f64(0.02, 0.4) for _ in range(16)]
        r = PyRng.seed_from_u64(seed)
        assert [int(x) for x in oracle.rng_gen_range_usize(seed, 0, 60, 16)] == \
            [r.gen_range_usize(0, 60) for _ in range(16)]


def test_random_guess_is_feasible_and_in_range(oracle):  # calibration.rs:131-141, 179-185
    for i in range(1, 64):
        g = oracle.random_guess(8, _splitmix64(12345 ^ i))
        v0, kappa, theta, sigma, rho, lam, mu_j, sigma_j = g
        assert 0.005 <= v0 < 0.5 and 0.3 <= kappa < 8.0 and 0.005 <= theta < 0.5
        assert 0.02 <= sigma < max(math.sqrt(2.0 * kappa * theta) * 0.9, 0.05)
        assert -0.9 <= rho < 0.9 and 0.0 <= lam < 2.0 and -0.3 <= mu_j < 0.1 and 0.02 <= sigma_j < 0.4
        assert 2.0 * kappa * theta > sigma * sigma or sigma < 0.05  # Feller by construction above the floor
        r = PyRng.seed_from_u64(_splitmix64(12345 ^ i))
        py = [r.gen_range_f64(0.005, 0.5), r.gen_range_f64(0.3, 8.0), r.gen_range_f64(0.005, 0.5)]
        cap = max(math.sqrt((2.0 * py[1]) * py[2]) * 0.9, 0.05)
        py += [r.gen_range_f64(0.02, cap), r.gen_range_f64(-0.9, 0.9), r.gen_range_f64(0.0, 2.0),
               r.gen_range_f64(-0.3, 0.1), r.gen_range_f64(0.02, 0.4)]
        assert list(g) == py


# ---- the reference's calibration tests, run on the oracle ------------------
TRUE_H = [0.04, 2.0, 0.04, 0.3, -0.5]
TRUE_B = TRUE_H + [0.5, -0.1, 0.15]
P0_H = [0.05, 1.5, 0.05, 0.4, -0.3]


def _make_quotes(oracle, p, bates=False):  # calibration.rs:980-1018
    rows, ivs = [], []
    for t in (0.25, 0.5, 1.0):
        for k in (80.0, 90.0, 95.0, 100.0, 105.0, 110.0, 120.0):
            ot = 0 if k >= 100.0 else 1
            px = (oracle.bates_price if bates else oracle.heston_price)(100.0, k, t, 0.03, 0.0, p, ot)
            c = oracle.contracts(100.0, k, t, 0.03, 0.0, ot, vol=0.2)
            iv = oracle.implied_vol(c, px)
            if iv is not None and 0.01 < iv < 2.0:
                rows.append(c[0])
                ivs.append(iv)
    return np.array(rows), np.array(ivs)


@pytest.fixture(scope="module")
def heston_quotes(oracle):
    return _make_quotes(oracle, TRUE_H)


@pytest.fixture(scope="module")
def bates_quotes(oracle):
    return _make_quotes(oracle, TRUE_B, bates=True)


def test_prune_mechanism_aborts_a_hopeless_restart(oracle, heston_quotes):  # calibration.rs:1180-1196
    con, iv = heston_quotes
    r = oracle.calibrate_ex(5, con, iv, [0.3, 7.5, 0.35, 0.12, 0.8], shared_best=1e-10)
    assert r["early_stopped"] and r["iters"] < 200 and not r["converged"]


def test_prune_mechanism_does_not_kill_a_competitive_restart(oracle, heston_quotes):  # calibration.rs:1198-1214
    con, iv = heston_quotes
    r = oracle.calibrate_ex(5, con, iv, P0_H, shared_best=float("inf"))
    assert not r["early_stopped"] and r["converged"] and r["rmse"] < 0.005


def test_multistart_beats_bad_single_start(oracle, heston_quotes):  # calibration.rs:1216-1234
    con, iv = heston_quotes
    bad = [0.25, 6.0, 0.3, 0.15, 0.6]
    single = oracle.calibrate(5, con, iv, bad)
    best, allr, n_conv, n_pruned, bi = oracle.calibrate_multistart(5, con, iv, bad, 8, 12345)
    assert n_conv >= 1
    assert best["rmse"] <= single["rmse"] + 1e-9
    assert best["rmse"] < 0.01
    assert allr[bi]["rmse"] == best["rmse"] and n_pruned == int(allr["early_stopped"].sum())


def test_de_global_recovers_heston_params(oracle, heston_quotes):  # calibration.rs:1073-1099
    con, iv = heston_quotes
    res, de_sse, pop, fit = oracle.calibrate_global(5, con, iv, 40, 60, 777)
    p = res["params"]
    assert res["rmse"] < 0.01 and abs(p[0] - 0.04) < 0.01 and abs(p[4] + 0.5) < 0.1
    assert 2.0 * p[1] * p[2] > p[3] * p[3]
    assert res["rmse"] <= math.sqrt(de_sse / iv.size) + 1e-9
    assert de_sse == fit.min() and pop.shape == (40, 5)


def test_de_global_bates_lands_where_the_reference_recorded(oracle, bates_quotes):  # calibration.rs:1101-1131
    con, iv = bates_quotes
    res, de_sse, pop, fit = oracle.calibrate_global(8, con, iv, 60, 80, 999)
    p = res["params"]
    assert res["rmse"] < 0.005 and 2.0 * p[1] * p[2] > p[3] * p[3] and p[0] > 0.0 and p[5] >= 0.0
    # "this run found params wildly different from the generating ones
    #  (v0=1.64 vs true 0.04, kappa=21 vs true 2, ...) with rmse essentially 0"
    assert round(p[0], 2) == 1.64 and round(p[1]) == 21
    # "Bates, DE, no p0: cond = inf"  (calibration.rs:937-976)
    assert res["condition_number"] > 1e10 or not math.isfinite(res["condition_number"])


def test_condition_numbers_match_the_recorded_runs(oracle, heston_quotes, bates_quotes):  # calibration.rs:941-976
    con, iv = heston_quotes
    h = oracle.calibrate(5, con, iv, P0_H)
    assert math.isfinite(h["condition_number"]) and abs(h["condition_number"] / 3.2e6 - 1.0) < 0.05
    con_b, iv_b = bates_quotes
    b = oracle.calibrate(8, con_b, iv_b, P0_H + [0.3, -0.05, 0.1])
    assert math.isfinite(b["condition_number"]) and abs(b["condition_number"] / 3.7e7 - 1.0) < 0.05


def test_regularization_does_not_hurt_a_well_identified_case(oracle, heston_quotes):  # calibration.rs:911-935
    con, iv = heston_quotes
    unreg = oracle.calibrate(5, con, iv, P0_H)
    reg = oracle.calibrate(5, con, iv, P0_H, prior=[0.045, 1.8, 0.045, 0.32, -0.45], reg_weight=1e-3)
    assert reg["rmse"] < 0.002 and abs(reg["params"][0] - unreg["params"][0]) < 0.005
    assert round(reg["rmse"], 4) == 0.0006  # "0.0006 vol points is nothing against real quote noise"


def test_regularization_recovers_plausible_params(oracle, bates_quotes):  # calibration.rs:870-909
    con, iv = bates_quotes
    prior = [0.035, 1.8, 0.04, 0.35, -0.45, 0.4, -0.08, 0.12]
    res, _, _, _ = oracle.calibrate_global(8, con, iv, 60, 80, 999, prior=prior, reg_weight=1e-3)
    p = res["params"]
    assert res["rmse"] < 0.005 and math.isfinite(res["condition_number"]) and res["condition_number"] < 1e9
    assert abs(p[0] - 0.04) < 0.01 and abs(p[1] - 2.0) < 0.5 and abs(p[5] - 0.5) < 0.15
    assert abs(p[6] + 0.1) < 0.05 and abs(p[7] - 0.15) < 0.05


def test_exact_jacobian_variant_reaches_the_same_fit(oracle, heston_quotes):
    con, iv = heston_quotes
    a = oracle.calibrate_ex(5, con, iv, P0_H, jac_mode=0)
    b = oracle.calibrate_ex(5, con, iv, P0_H, jac_mode=1)
    assert a["converged"] and b["converged"]
    assert np.allclose(a["params"][:5], b["params"][:5], rtol=1e-7, atol=1e-9)
    assert abs(a["condition_number"] / b["condition_number"] - 1.0) < 1e-4
