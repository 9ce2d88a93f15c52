#!/usr/bin/env python
"""Benchmark of the Heston/Bates CF pricing path on B200.

One step = one pass of the hot path over one batch: the 1,048,576-contract
Bates deep-wing batch (4096 surfaces x 256 contracts, tol 1e-10) priced by
the persistent multi-surface kernel.  Prints ONE JSON line (rank 0).

  value      contracts/s, inputs resident in HBM, CUDA events on the launch
             stream; L2 flushed (512 MiB write) before every step.
  e2e        same metric through the public host API (pinned host buffers,
             H2D of the step's contracts/params/offsets and D2H of prices
             inside the timed region, wall clock around the synchronous call).
  e2e_pageable  the same from pageable host buffers (what a Rust Vec caller
             passes): the library copies contracts in and prices out.
  parity     worst |price - oracle| / S over a sample; above 1e-9 the run
             prints its line and exits with status 3.
  plain      the reference-shaped drop-in: one batch_bates call per surface
             (host buffers, synchronous), on a sample of surfaces.
  roofline   FP64 bound: algorithmic FP64 ops per launch (ope_b200.roofline)
             / average launch time vs the measured DFMA peak of this GPU.
  cpu_baseline  the CPU oracle (the reference restated in C++, OpenMP over
             all host cores) on a bounded sample of the same workload.

``--impl reference`` times that CPU implementation alone (rank 0 only).
Multi-GPU (torchrun): every rank prices its own 1M-contract shard (weak
scaling, no collective on the data path); timing is the max over ranks.
``--gpus N`` without torchrun starts the N ranks itself; under torchrun
WORLD_SIZE must equal N.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "options-pricing-engine-rs_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Heston/Bates prices/s batched vs plain, 1 B200, ≤1e-9 err; p50/p99 latency"
UNIT = "contracts/s"
PARITY_BAR = 1e-9  # max |price - oracle| / S per contract; the run exits 3 above it


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--contracts", type=int, default=1 << 20, help="contracts per rank")
    ap.add_argument("--plain-surfaces", type=int, default=256)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-calib", action="store_true", help="skip the config-4 calibration section")
    ap.add_argument("--no-gradient", action="store_true", help="skip the adjoint-gradient section")
    ap.add_argument("--grad-n", type=int, default=1 << 18, help="contracts in the adjoint-gradient section")
    ap.add_argument("--no-serving", action="store_true", help="skip the config-5 serving section")
    ap.add_argument("--serving-rates", default="100,1000,5000,10000,15000,20000")
    ap.add_argument("--serving-seconds", type=float, default=10.0, help="seconds of arrivals per serving rate")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape (no ope_autotune)")
    ap.add_argument("--no-grid", action="store_true", help="skip the grid-surface (config-2 layout) section")
    ap.add_argument("--grid-only", action="store_true",
                    help="run only the grid-surface section (1 GPU) and print its JSON object")
    return ap.parse_args()


def workload(n: int, rank: int):
    from ope_b200 import workloads as W
    from ope_b200.multi import shard_seed

    return W.c3(n=n, per_surface=256, seed=shard_seed(3, rank))


def config_of(w, world: int) -> dict:
    return {
        "workload": w.name if world == 1 else w.name + "-per-rank",
        "model": "bates",
        "n_contracts": w.n,
        "n_surfaces": w.n_surf,
        "contracts_per_surface": 256,
        "tol": w.tol,
        "max_panels": 200,
        "parallelism": "replicas" if world > 1 else "single-gpu",
        "l2": "flushed between timed steps (512 MiB device write); inputs 59 MB < L2",
    }


# ----------------------------------------------------------------- CPU side
def cpu_sample(w, seconds: float, rng_seed: int = 0, gpu_prices=None):
    """Time the oracle (all host cores) on a random contract sample sized to ~`seconds`.

    With gpu_prices (the GPU's prices for the whole workload) also returns the
    worst |gpu - oracle| over the sample: the per-contract parity check."""
    from oracle import oracle as O

    O.build()
    rng = np.random.default_rng(rng_seed)
    si = w.surf_idx()
    probe = np.sort(rng.choice(w.n, 2048, replace=False))
    t0 = time.perf_counter()
    O.batch_price(w.contracts[probe], w.params, True, w.tol, surf_idx=si[probe])
    rate = probe.size / (time.perf_counter() - t0)
    m = int(min(w.n, max(2048, rate * seconds)))
    idx = np.sort(rng.choice(w.n, m, replace=False))
    t0 = time.perf_counter()
    ref = O.batch_price(w.contracts[idx], w.params, True, w.tol, surf_idx=si[idx])
    dt = time.perf_counter() - t0
    if gpu_prices is not None:
        err = np.abs(gpu_prices[idx] - ref) / w.contracts["spot"][idx]
        return m / dt, m, dt, O.max_threads(), float(err.max())
    return m / dt, m, dt, O.max_threads()


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    w = workload(args.contracts, 0)
    per_step = max(0.2, min(args.cpu_seconds, 60.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_sample(w, per_step / 4, rng_seed=17)
    rates, total_m, total_t, cores = [], 0, 0.0, 1
    for k in range(args.steps):
        rate, m, dt, cores = cpu_sample(w, per_step, rng_seed=100 + k)
        rates.append(rate)
        total_m += m
        total_t += dt
    value = total_m / total_t
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(w, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{total_m} random contracts of the workload over {args.steps} steps "
                                   f"(~{per_step:.0f} s each), OpenMP dynamic schedule, C++ restatement "
                                   f"of the reference (no Rust toolchain on this box)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,uuid,utilization.gpu,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.uuid:
            cmd[1:1] = ["-i", self.uuid]
        try:
            self.p = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.f.read())) if len(r) >= 11]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                util, clk, mx = float(r[2]), float(r[3]), float(r[4])
            except ValueError:
                continue
            smax = mx
            if util >= 50:
                sm.append(clk)
                for nm, v in zip(names, r[7:11]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples_under_load": len(sm)}


def bench_calibration(args) -> dict:
    """Config 4: 256 Heston surfaces x 300 quotes, LM in IV space on the device
    (one conditional-WHILE graph), against the reference's LM (the oracle:
    finite-difference Jacobian, calibration.rs:433-569) on the host cores."""
    import ope_b200 as ope
    from ope_b200 import workloads as W

    def price_fn(con, params, sidx):
        off = np.concatenate([[0], np.cumsum(np.bincount(sidx, minlength=params.shape[0]))])
        return ope.price_surfaces(ope.MODEL_HESTON, con, off, params, tol=1e-10)

    con, iv, off, true_p, p0 = W.c4(price_fn, ope.batch_implied_vol)
    ope.calibrate_surfaces(ope.MODEL_HESTON, con, iv, off, p0)  # builds the graph
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        r = ope.calibrate_surfaces(ope.MODEL_HESTON, con, iv, off, p0)
        ts.append(time.perf_counter() - t0)
    n_surf = off.size - 1
    out = {
        "workload": "c4-heston-256-surfaces-30x10-noise0.005", "quotes": int(con.size), "surfaces": int(n_surf),
        "value": n_surf / min(ts), "unit": "surfaces/s", "ms": 1e3 * min(ts),
        "iters_mean": float(r["iters"].mean()), "iters_max": int(r["iters"].max()),
        "stopped_converged": int((r["status"] == 1).sum()), "stopped_damping_cap": int((r["status"] == 2).sum()),
        "stopped_iteration_cap": int((r["status"] == 3).sum()), "rmse_median": float(np.median(r["rmse"])),
        "jacobian": "adjoint kernel / BSM vega (exact)", "loop": "one CUDA graph launch (conditional WHILE node)",
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        O.build()
        k = max(2, min(O.max_threads(), 8))
        t0 = time.perf_counter()
        ro = O.calibrate_many(5, con[:off[k]], iv[:off[k]], off[:k + 1], p0[:k])
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": k / dt, "unit": "surfaces/s", "cores": min(k, O.max_threads()),
                               "kind": "port", "sample": f"{k} surfaces, reference LM with FD Jacobian, "
                                                         f"one surface per thread, {dt:.1f} s",
                               "rmse_max_abs_diff_vs_gpu": float(np.max(np.abs(ro["rmse"] - r["rmse"][:k])))}
    out["multistart"] = bench_multistart(args, con, iv, off, p0)
    out["global"] = bench_global(args, con, iv, off)
    return out


def bench_multistart(args, con, iv, off, p0, n_surf=64, n_restarts=8, seed=12345) -> dict:
    """calibration.rs:246-314 on the first n_surf config-4 surfaces: every
    restart of every surface one LM state machine of one device graph, restarts
    of a surface pruning against their shared best."""
    import ope_b200 as ope

    o = off[:n_surf + 1]
    c, v = con[:o[-1]], iv[:o[-1]]
    ope.calibrate_multistart(ope.MODEL_HESTON, c, v, o, p0[:n_surf], n_restarts, seed)  # builds the graph
    t0 = time.perf_counter()
    r = ope.calibrate_multistart(ope.MODEL_HESTON, c, v, o, p0[:n_surf], n_restarts, seed)
    dt = time.perf_counter() - t0
    out = {"surfaces": n_surf, "restarts": n_restarts, "value": n_surf / dt, "unit": "surfaces/s", "ms": 1e3 * dt,
           "pruned_per_surface": float(r["n_pruned"].mean()), "converged_per_surface": float(r["n_converged"].mean()),
           "best_rmse_median": float(np.median(r["best"]["rmse"]))}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        t0 = time.perf_counter()
        best, _, _, _, _ = O.calibrate_multistart(5, con[:off[1]], iv[:off[1]], p0[0], n_restarts, seed)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "surfaces/s", "cores": O.max_threads(), "kind": "port",
                               "sample": f"1 surface, {n_restarts} restarts in lockstep over the host cores, "
                                         f"reference LM (FD Jacobian), {dt:.1f} s",
                               "best_rmse_abs_diff_vs_gpu": float(abs(best["rmse"] - r["best"]["rmse"][0]))}
    return out


def bench_global(args, con, iv, off, n_surf=16, n_pop=40, n_gen=60, seed=777) -> dict:
    """calibration.rs:316-427 (DE/rand/1/bin + LM polish) on the first n_surf
    config-4 surfaces: each generation prices every member of every surface
    in one persistent launch; the generation loop is one device graph."""
    import ope_b200 as ope

    o = off[:n_surf + 1]
    c, v = con[:o[-1]], iv[:o[-1]]
    ope.calibrate_global(ope.MODEL_HESTON, c[:o[1]], v[:o[1]], o[:2], n_pop, 1, seed)  # warm
    t0 = time.perf_counter()
    r = ope.calibrate_global(ope.MODEL_HESTON, c, v, o, n_pop, n_gen, seed)
    dt = time.perf_counter() - t0
    pricings = int(o[-1]) * n_pop * (n_gen + 1)
    out = {"surfaces": n_surf, "n_pop": n_pop, "n_gen": n_gen, "value": n_surf / dt, "unit": "surfaces/s",
           "ms": 1e3 * dt, "member_pricings": pricings, "member_pricings_per_s": pricings / dt,
           "rmse_median": float(np.median(r["best"]["rmse"]))}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        t0 = time.perf_counter()
        ro, sse, _, _ = O.calibrate_global(5, con[:off[1]], iv[:off[1]], n_pop, n_gen, seed)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "surfaces/s", "cores": O.max_threads(), "kind": "port",
                               "sample": f"1 surface, population over the host cores, reference LM polish, "
                                         f"{dt:.1f} s",
                               "de_best_sse_rel_diff_vs_gpu": float(abs(sse - r["de_best_sse"][0]) / sse)}
    return out


def bench_gradient(args, w, dev, flush, stream, price_kernel_ms) -> dict:
    """Prices + d price / d(v0, kappa, theta, sigma, rho, lambda, mu_j, sigma_j)
    by the reverse-mode adjoint kernel (ad.rs:695-731, 882-895) on the first
    grad_n contracts of the pricing workload, device-resident, L2 flushed,
    CUDA events; checked against the oracle's forward-mode AD on a sample."""
    import torch

    import ope_b200 as ope

    n_surf = int(np.searchsorted(w.surf_offsets, min(args.grad_n, w.n), side="right") - 1)
    n = int(w.surf_offsets[n_surf])
    d_con = torch.from_numpy(w.contracts[:n].view(np.uint8).copy()).to(dev)
    d_off = torch.from_numpy(w.surf_offsets[:n_surf + 1].copy()).to(dev)
    d_par = torch.from_numpy(w.params[:n_surf].copy()).to(dev)
    d_px = torch.empty(n, dtype=torch.float64, device=dev)
    d_g = torch.empty((n, 8), dtype=torch.float64, device=dev)

    def step():
        ope.price_gradient_surfaces_device(ope.MODEL_BATES, d_con, n, d_off, n_surf, d_par, d_px, d_g, tol=w.tol,
                                           stream=stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    k_ms = statistics.mean(ms)
    out = {"workload": f"c3-bates-deepwing first {n} contracts ({n_surf} surfaces)", "n_contracts": n,
           "params_per_contract": 8, "value": n / (k_ms * 1e-3), "unit": "contracts/s (price + 8-parameter gradient)",
           "kernel_ms": k_ms, "cost_vs_price": (k_ms / n) / (price_kernel_ms / w.n)}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        rng = np.random.default_rng(7)
        pick = np.sort(rng.choice(n, 2000, replace=False))
        sidx = (np.searchsorted(w.surf_offsets, pick, side="right") - 1).astype(np.int32)
        t0 = time.perf_counter()
        price, grad = O.batch_price_gradient(w.contracts[pick], w.params, True, w.tol, surf_idx=sidx)
        dt = time.perf_counter() - t0
        g = d_g.cpu().numpy()[pick]
        # relative error with an absolute floor of 1e-9 S per component (the adjoint tests' bar)
        lim = 1e-7 * np.abs(grad) + 1e-9 * w.contracts["spot"][pick, None]
        worst = float((np.abs(g - grad) / lim).max())
        out["cpu_baseline"] = {"value": pick.size / dt, "unit": out["unit"], "cores": O.max_threads(),
                               "kind": "port", "sample": f"{pick.size} contracts, forward-mode AD, 8 passes each, "
                                                         f"{dt:.1f} s"}
        out["parity"] = {"worst_err_over_bar": worst, "bar": "1e-7 relative + 1e-9 S absolute, per component",
                         "against": "oracle forward-mode AD (ad.rs:695-731, 882-895)",
                         "max_abs_price_err_over_spot": float(np.max(np.abs(d_px.cpu().numpy()[pick] - price)
                                                                     / w.contracts["spot"][pick]))}
    return out


def bench_greeks(args, w, dev, flush, stream) -> dict:
    """greeks.rs:19-72 (bump-and-reprice, 14 pricings per contract) and
    ad.rs:736-865 (AD Greeks: 9 pricings + 3 adjoint evaluations per contract)
    on 65,536 contracts of the pricing workload under one parameter set
    (surface 0's), device-resident, L2 flushed, CUDA events."""
    import ctypes

    import torch

    import ope_b200 as ope

    n = min(65536, w.n)
    con = w.contracts[:n]
    par = w.params[0]
    d_con = torch.from_numpy(con.view(np.uint8).copy()).to(dev)
    d_par = torch.from_numpy(par.copy()).to(dev)
    d_out = torch.empty(n * 8, dtype=torch.float64, device=dev)
    lib = ope._lib.load()

    def run(fn, flags=0):
        o = ope._lib.Options(tol=w.tol, flags=ope._lib.FLAG_DEVICE_PTRS | flags, reserved=0,
                             stream=stream.cuda_stream)
        ope._lib.check(fn(ope.MODEL_BATES, d_con.data_ptr(), n, d_par.data_ptr(), d_out.data_ptr(),
                          ctypes.byref(o)))

    out = {"workload": f"c3-bates-deepwing first {n} contracts, surface 0's parameters", "n_contracts": n}
    for name, fn, flags in (("bump", lib.ope_batch_greeks_ex, 0), ("ad", lib.ope_batch_greeks_ad, 0),
                            ("analytic", lib.ope_batch_greeks_ad, ope._lib.FLAG_ANALYTIC_GREEKS)):
        for _ in range(max(args.warmup, 3)):
            flush.zero_()
            run(fn, flags)
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run(fn, flags)
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        out[name] = {"value": n / (statistics.mean(ms) * 1e-3), "unit": "contracts/s (8 Greeks each)",
                     "ms": statistics.mean(ms)}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        rng = np.random.default_rng(5)
        pick = np.sort(rng.choice(n, 512, replace=False))
        t0 = time.perf_counter()
        ref = O.batch_greeks(con[pick], par, True, tol=w.tol)
        dt = time.perf_counter() - t0
        bump = ope.batch_bates_greeks(con[pick], par, tol=w.tol)
        out["bump"]["cpu_baseline"] = {"value": pick.size / dt, "unit": out["bump"]["unit"], "cores": O.max_threads(),
                                       "kind": "port", "sample": f"{pick.size} contracts, {dt:.1f} s"}
        out["bump"]["max_abs_price_err_over_spot"] = float(np.max(np.abs(bump["price"] - ref[:, 0])) / 100.0)
        t0 = time.perf_counter()
        refad = np.array([O.greeks_ad(c, par, True, w.tol) for c in con[pick[:64]]])
        dt = time.perf_counter() - t0
        ad = ope.batch_greeks_ad(ope.MODEL_BATES, con[pick[:64]], par, tol=w.tol)
        out["ad"]["cpu_baseline"] = {"value": 64 / dt, "unit": out["ad"]["unit"], "cores": 1, "kind": "port",
                                     "sample": f"64 contracts, one thread, {dt:.1f} s"}
        out["ad"]["max_abs_vega_rel_err"] = float(np.max(np.abs(ad["vega"] - refad[:, 3]) / np.abs(refad[:, 3])))
        an = ope.batch_greeks_ad(ope.MODEL_BATES, con[pick[:64]], par, tol=w.tol, analytic=True)
        out["analytic"]["max_abs_vega_rel_err"] = float(np.max(np.abs(an["vega"] - refad[:, 3])
                                                               / np.abs(refad[:, 3])))
        out["analytic"]["cpu_baseline"] = out["ad"]["cpu_baseline"]
    out["analytic"]["what"] = ("all eight Greeks as exact derivatives: one pricing + one backward pass of seven "
                               "derivative integrals (OPE_FLAG_ANALYTIC_GREEKS)")
    return out


def bench_implied_vol(args, w, dev, flush, stream, d_con, d_prices, prices) -> dict:
    """batch.rs:51-56 / iv.rs:14-83 on the device: Black-Scholes implied vols of
    the headline batch's 1M Bates prices (device-resident, L2 flushed, CUDA
    events), against the oracle's restatement on the host cores."""
    import ctypes

    import torch

    import ope_b200 as ope

    n = w.n
    d_iv = torch.empty(n, dtype=torch.float64, device=dev)
    d_ok = torch.empty(n, dtype=torch.int32, device=dev)
    lib = ope._lib.load()
    o = ope._lib.Options(tol=w.tol, flags=ope._lib.FLAG_DEVICE_PTRS, reserved=0, stream=stream.cuda_stream)

    def run():
        ope._lib.check(lib.ope_batch_implied_vol(d_con.data_ptr(), n, d_prices.data_ptr(), d_iv.data_ptr(),
                                                 d_ok.data_ptr(), ctypes.byref(o)))

    for _ in range(max(args.warmup, 3)):
        flush.zero_()
        run()
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        run()
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    iv, ok = d_iv.cpu().numpy(), d_ok.cpu().numpy().astype(bool)
    out = {"workload": f"c3-bates-deepwing-{n} prices -> Black-Scholes implied vols", "n_contracts": n,
           "value": n / (statistics.mean(ms) * 1e-3), "unit": "contracts/s", "ms": statistics.mean(ms),
           "solved_fraction": float(ok.mean())}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        rng = np.random.default_rng(9)
        pick = np.sort(rng.choice(n, min(n, 200000), replace=False))
        t0 = time.perf_counter()
        riv, rok = O.batch_implied_vol(w.contracts[pick], prices[pick])
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": pick.size / dt, "unit": "contracts/s", "cores": O.max_threads(),
                               "kind": "port", "sample": f"{pick.size} contracts, {dt:.2f} s"}
        # Where the time value is below 1e-9 S the price is intrinsic to the last ulps and
        # the IV is not identifiable in double precision; elsewhere both solvers stop at
        # |price error| < 1e-10 (iv.rs:69), so each IV is known to 1e-10 / vega.
        c = w.contracts[pick]
        eq, er = np.exp(-c["div_yield"] * c["expiry"]), np.exp(-c["rate"] * c["expiry"])
        intr = np.where(c["opt_type"] == 0, np.maximum(c["spot"] * eq - c["strike"] * er, 0.0),
                        np.maximum(c["strike"] * er - c["spot"] * eq, 0.0))
        well = (prices[pick] - intr) > 1e-9 * c["spot"]
        both = well & rok & ok[pick]
        with np.errstate(all="ignore"):
            vt = riv * np.sqrt(c["expiry"])
            d1 = (np.log(c["spot"] / c["strike"]) + (c["rate"] - c["div_yield"] + 0.5 * riv * riv) * c["expiry"]) / vt
            vega = c["spot"] * eq * np.exp(-0.5 * d1 * d1) / np.sqrt(2 * np.pi) * np.sqrt(c["expiry"])
            lim = 2.5e-10 / np.maximum(vega, 1e-300) + 1e-12
        out["parity"] = {"well_identified": int(well.sum()),
                         "same_solvability_where_identified": bool(np.array_equal(rok[well], ok[pick][well])),
                         "worst_iv_err_over_bar": float(np.max(np.abs(iv[pick][both] - riv[both]) / lim[both]))
                         if both.any() else 0.0,
                         "bar": "2.5e-10 / vega (both solvers stop at |price error| < 1e-10, iv.rs:69)",
                         "against": "oracle restatement of iv.rs:14-83 (Halley, bisection fallback)"}
    return out


def bench_grid_surfaces(args, dev, flush, stream) -> dict:
    """Surfaces laid out expiry by expiry (the uneven strike x expiry grids of
    config 2, 4096 surfaces, ~1.46M contracts; Heston, and the same grids with
    Bates parameters): the strikes of one expiry share the characteristic
    function per panel in the run kernel.  Kernel time of the automatic launch
    (a device probe picks the run kernel and its contracts per unit) against
    one contract per unit, bit-identity of the two, and the oracle on a
    sample."""
    import torch

    import ope_b200 as ope
    from ope_b200 import workloads as W
    from oracle import oracle as O

    saved = {m: ope.tune_table(m)[0] for m in (ope.MODEL_HESTON, ope.MODEL_BATES)}
    base = W.c2()
    rng = np.random.default_rng(9)
    ns = base.params.shape[0]
    bates_params = np.concatenate([base.params, rng.uniform(0, 1.5, (ns, 1)), rng.uniform(-0.3, 0.1, (ns, 1)),
                                   rng.uniform(0.05, 0.4, (ns, 1))], axis=1)
    out = {"what": "config-2 grids (expiry-major): automatic launch (run probe -> run kernel) vs one contract per "
                   "unit, device buffers, L2 flushed between steps", "unit": UNIT}
    try:
        for name, model, params in (("heston", ope.MODEL_HESTON, base.params), ("bates", ope.MODEL_BATES, bates_params)):
            d_con = torch.from_numpy(base.contracts.view(np.uint8).copy()).to(dev)
            d_off = torch.from_numpy(base.surf_offsets.copy()).to(dev)
            d_par = torch.from_numpy(np.ascontiguousarray(params)).to(dev)
            res, prices = {}, {}
            for mode, pu in (("automatic", 0), ("one_contract_per_unit", 1)):
                rows = [dict(r, per_unit=pu) for r in saved[model]]
                ope.set_tune_table(model, rows)
                d_out = torch.full((base.n,), float("nan"), dtype=torch.float64, device=dev)
                ms = []
                for i in range(args.warmup + args.steps):
                    flush.zero_()
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    ope.price_surfaces_device(model, d_con, base.n, d_off, base.n_surf, d_par, d_out, tol=base.tol,
                                              stream=stream.cuda_stream)
                    b.record(stream)
                    torch.cuda.synchronize()
                    if i >= args.warmup:
                        ms.append(a.elapsed_time(b))
                per_unit = ope.last_per_unit()
                prices[mode] = d_out.cpu().numpy()
                res[mode] = {"kernel_ms": float(np.mean(ms)), "value": base.n / (np.mean(ms) * 1e-3),
                             "contracts_per_unit": per_unit}
            res["speedup"] = res["one_contract_per_unit"]["kernel_ms"] / res["automatic"]["kernel_ms"]
            res["bit_identical"] = bool(np.array_equal(prices["automatic"].view(np.int64),
                                                       prices["one_contract_per_unit"].view(np.int64)))
            pick = np.sort(np.random.default_rng(3).choice(base.n, 400, replace=False))
            orc = O.batch_price(base.contracts[pick], params, model == ope.MODEL_BATES, base.tol,
                                surf_idx=base.surf_idx()[pick])
            res["max_abs_err_over_spot"] = float(np.max(np.abs(prices["automatic"][pick] - orc)) / 100.0)
            res["n_contracts"] = int(base.n)
            out[name] = res
    finally:
        for m, rows in saved.items():
            ope.set_tune_table(m, rows)
    return out


def bench_serving(args, tuned: bool) -> dict:
    """Config 5: Poisson arrivals, 80 % Bates surface reprices / 20 % Heston
    calibrations, sizes log-uniform in [20, 2000] contracts.  For every offered
    rate a fresh stream with --serving-seconds of arrivals (contents drawn from
    a pool of 3,000 distinct requests), then up to 20 s to drain; latencies
    over the steady half of the arrivals.  The highest offered rate whose
    reprices all finish and whose reprice latency does not grow across the
    run is reported as the sustained reprice rate.  With the autotuner on, the
    5,000 req/s stream is run once more with the default launch shape."""
    import ope_b200 as ope
    from ope_b200 import serving as SV

    out = {"mix": "80% Bates reprice / 20% Heston calibration, sizes log-uniform [20, 2000]",
           "seconds_of_arrivals_per_rate": args.serving_seconds, "rates": []}
    pool = SV.make_stream(3000, seed=5)
    with SV.Server(hbm_fraction=0.25, max_inflight=4) as srv:
        # warm: a few requests of each kind
        for r in pool[:16]:
            rid = srv.submit_price(1, r.contracts, r.params) if r.kind == 0 else srv.submit_calibrate(
                0, r.contracts, r.iv, r.params)
            srv.wait(rid)
        sustained = None
        for rate in [float(x) for x in args.serving_rates.split(",")]:
            res = SV.run_sustained(srv, pool, rate, args.serving_seconds, seed=int(rate))
            row = SV.summarize_sustained(res)
            out["rates"].append(row)
            if row["reprice_sustained"]:
                sustained = rate
        out["highest_offered_rate_with_reprices_sustained"] = sustained
        if tuned:
            ope.set_autotune(False)
            res = SV.run_sustained(srv, pool, 5000.0, min(5.0, args.serving_seconds), seed=5000)
            ope.set_autotune(True)
            out["default_launch_shape_at_5000_req_per_s"] = SV.summarize_sustained(res)
        st = srv.stats()
    out["server"] = {k: st[k] for k in ("batches", "batched_requests", "max_inflight", "rejected",
                                         "hbm_budget_bytes", "hbm_peak_bytes")}
    return out


def nodes_percentiles(nb) -> dict:
    """Integrand evaluations per contract (both integrals: 15 (1 + 2 bisections)
    each) as percentiles over the batch; the load imbalance the work queue absorbs."""
    nodes = 15 * (1 + 2 * nb.reshape(-1, 2).astype(np.int64)).sum(axis=1)
    return {"p50": float(np.percentile(nodes, 50)), "p90": float(np.percentile(nodes, 90)),
            "p99": float(np.percentile(nodes, 99)), "max": int(nodes.max()),
            "integrals_at_panel_cap": int((nb >= 199).sum())}


def read_traffic():
    p = os.path.join(ROOT, "profiles", "c3_persistent_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch_full")
    return None


# ----------------------------------------------------------------- GPU side
def run_ours(args) -> None:
    import torch

    import ope_b200 as ope
    from ope_b200 import roofline

    from ope_b200 import multi

    rank, local_rank, world = multi.rank_info()
    if torch.cuda.device_count() < world:
        raise SystemExit(f"bench.py: {world} ranks but {torch.cuda.device_count()} visible GPU(s)")
    torch.cuda.set_device(local_rank)
    dist = multi.init("nccl")

    def barrier():
        multi.barrier(dist)

    def max_over_ranks(x: float) -> float:
        return multi.max_over_ranks(dist, x, device="cuda")

    w = workload(args.contracts, rank)
    n, n_surf = w.n, w.n_surf
    model = ope.MODEL_BATES
    dev = torch.device("cuda", local_rank)
    d_con = torch.from_numpy(w.contracts.view(np.uint8).copy()).to(dev)
    d_off = torch.from_numpy(w.surf_offsets).to(dev)
    d_par = torch.from_numpy(w.params.copy()).to(dev)
    d_out = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    # untimed set-up: the launch-shape autotuner (ope_autotune) measures this
    # device once; every call below uses its table unless --no-autotune
    tune = None
    if not args.no_autotune:
        t0 = time.perf_counter()
        rows = ope.autotune(model)
        tune = {"seconds": time.perf_counter() - t0, "table": rows}

    # untimed: per-integral bisection counts for the work tally
    nb = np.zeros(2 * n, np.int32)
    ope.price_surfaces(model, w.contracts, w.surf_offsets, w.params, tol=w.tol, bisections=nb)
    flops_per_launch = roofline.work_flops(nb, True)

    def step():
        ope.price_surfaces_device(model, d_con.data_ptr(), n, d_off.data_ptr(), n_surf, d_par.data_ptr(),
                                  d_out.data_ptr(), tol=w.tol, stream=stream.cuda_stream)

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_all0, t_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    launches0 = ope.kernel_launch_count()
    t_all0.record(stream)
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    t_all1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = ope.kernel_launch_count() - launches0
    region_ms = max_over_ranks(t_all0.elapsed_time(t_all1))
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    kern_avg = statistics.mean(kern_ms)
    value = multi.weak_scaling_value(world, n, args.steps, region_ms * 1e-3)

    # check this run's prices against the stats run (same bits expected)
    ref_prices = np.empty(n)
    ope.price_surfaces(model, w.contracts, w.surf_offsets, w.params, tol=w.tol, out=ref_prices)
    assert np.array_equal(d_out.cpu().numpy(), ref_prices), "device-path prices differ from host-path prices"

    # e2e through the public API with pinned host buffers
    pin_con = torch.empty(n * 56, dtype=torch.uint8, pin_memory=True).numpy().view(w.contracts.dtype)
    pin_con[:] = w.contracts
    pin_off = torch.empty(n_surf + 1, dtype=torch.int64, pin_memory=True).numpy()
    pin_off[:] = w.surf_offsets
    pin_par = torch.empty((n_surf, 8), dtype=torch.float64, pin_memory=True).numpy()
    pin_par[:] = w.params
    pin_out = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    for _ in range(max(1, args.warmup)):
        ope.price_surfaces(model, pin_con, pin_off, pin_par, tol=w.tol, out=pin_out)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ope.price_surfaces(model, pin_con, pin_off, pin_par, tol=w.tol, out=pin_out)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    clk = clocks.stop()  # sampled over both timed regions (device and e2e)
    barrier()
    e2e_value = multi.weak_scaling_value(world, n, args.steps, e2e_s)
    h2d = n * 56 + (n_surf + 1) * 8 + n_surf * 8 * 8
    d2h = n * 8

    # e2e from pageable host buffers (a Rust Vec): the library stages the
    # contracts into device memory and copies the prices back around the launch
    pg_out = np.empty(n)
    ope.price_surfaces(model, w.contracts, w.surf_offsets, w.params, tol=w.tol, out=pg_out)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ope.price_surfaces(model, w.contracts, w.surf_offsets, w.params, tol=w.tol, out=pg_out)
    pageable_s = max_over_ranks(time.perf_counter() - t0)
    pageable_value = multi.weak_scaling_value(world, n, args.steps, pageable_s)
    assert np.array_equal(pg_out, ref_prices), "pageable-buffer prices differ from the device-path prices"

    # the plain drop-in: one synchronous batch_bates call per surface (host buffers)
    rng = np.random.default_rng(1000 + rank)
    picks = np.sort(rng.choice(n_surf, min(args.plain_surfaces, n_surf), replace=False))

    def plain_run():
        for s in picks[:8]:
            ope.batch_bates(w.contracts[w.surf_offsets[s]:w.surf_offsets[s + 1]], w.params[s], tol=w.tol)
        barrier()
        t0 = time.perf_counter()
        cnt, call_ms = 0, []
        for s in picks:
            c = w.contracts[w.surf_offsets[s]:w.surf_offsets[s + 1]]
            t1 = time.perf_counter()
            ope.batch_bates(c, w.params[s], tol=w.tol)
            call_ms.append(1e3 * (time.perf_counter() - t1))
            cnt += c.size
        return world * cnt / max_over_ranks(time.perf_counter() - t0), call_ms

    # 2,048-contract calls (8 surfaces each, the size of a large serving request)
    groups = [list(range(8 * g, 8 * g + 8)) for g in range(0, min(64, n_surf // 8))]
    subs = [w.subset(g) for g in groups]

    def mid_run():
        for sub in subs[:4]:
            ope.price_surfaces(model, sub.contracts, sub.surf_offsets, sub.params, tol=w.tol)
        ms = []
        for sub in subs:
            t1 = time.perf_counter()
            ope.price_surfaces(model, sub.contracts, sub.surf_offsets, sub.params, tol=w.tol)
            ms.append(1e3 * (time.perf_counter() - t1))
        return ms

    def pct(ms):
        return {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))}

    plain_value, call_ms = plain_run()
    mid_ms = mid_run()
    shapes = None
    if tune is not None:  # the same calls with the default launch shape
        ope.set_autotune(False)
        plain_default, call_ms_default = plain_run()
        mid_ms_default = mid_run()
        ope.set_autotune(True)
        shapes = {"plain_value_default_shape": plain_default,
                  "latency_ms_per_256_contract_surface_default_shape": pct(call_ms_default),
                  "latency_ms_per_2048_contract_call": pct(mid_ms),
                  "latency_ms_per_2048_contract_call_default_shape": pct(mid_ms_default)}

    peak_flops, _ = ope.measure_fp64_peak()
    achieved = flops_per_launch / (kern_avg * 1e-3)
    traffic = read_traffic()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": region_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(w, world),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "ope_price_surfaces (host pointers, pinned: the kernel reads the contracts and writes the prices "
                       "in place over PCIe, zero-copy)"},
        "e2e_pageable": {"value": pageable_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                         "api": "ope_price_surfaces (host pointers, pageable: contracts copied to device memory before "
                                "the launch, prices copied back after it)"},
        "plain": {"value": plain_value, "unit": UNIT, "surfaces_sampled": int(picks.size),
                  "api": "ope_batch_bates per surface (host pointers, synchronous)",
                  "batched_e2e_over_plain": e2e_value / plain_value,
                  "latency_ms_per_256_contract_surface": pct(call_ms)},
        "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak_flops / 1e12, "unit": "TFLOP/s",
                     "frac": achieved / peak_flops, "traffic": traffic,
                     "peak_source": "measured DFMA-chain probe on this GPU (ope_measure_fp64_peak)",
                     "work": f"{flops_per_launch:.4e} FP64 ops per launch = nodes x F_node "
                             f"(F_node {roofline.F_NODE[(True, True)]}/{roofline.F_NODE[(True, False)]} P1/P2); "
                             f"nodes/contract {roofline.nodes_total(nb) / n:.1f}",
                     "kernel_ms": kern_avg,
                     "nodes_per_contract": nodes_percentiles(nb)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if tune is not None:
        tune.update(shapes or {})
        line["autotune"] = tune
    else:
        line["plain"]["latency_ms_per_2048_contract_call"] = pct(mid_ms)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, m, dt, cores, worst = cpu_sample(w, args.cpu_seconds, gpu_prices=ref_prices)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{m} random contracts of the workload in {dt:.1f} s",
                                "host_cpus_available": len(os.sched_getaffinity(0))}
        line["parity"] = {"max_abs_err_over_spot": worst, "bar": 1e-9, "contracts_checked": m,
                          "against": "CPU oracle (the reference restated), same tolerance, same contracts"}
    if rank == 0 and world == 1 and not args.no_gradient:
        line["gradient"] = bench_gradient(args, w, dev, flush, stream, kern_avg)
    if rank == 0 and world == 1 and not args.no_gradient:
        line["greeks"] = bench_greeks(args, w, dev, flush, stream)
    if rank == 0 and world == 1 and not args.no_gradient:
        line["implied_vol"] = bench_implied_vol(args, w, dev, flush, stream, d_con, d_out, ref_prices)
    if rank == 0 and world == 1 and not args.no_grid:
        line["grid_surfaces"] = bench_grid_surfaces(args, dev, flush, stream)
    if rank == 0 and world == 1 and not args.no_calib:
        line["calibration"] = bench_calibration(args)
    if rank == 0 and world == 1 and not args.no_serving:
        line["serving"] = bench_serving(args, tune is not None)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    worst = line.get("parity", {}).get("max_abs_err_over_spot", 0.0)
    if not worst <= PARITY_BAR:
        print(f"bench.py: parity breach: max |gpu - oracle| / S = {worst:.3e} > {PARITY_BAR:g}", file=sys.stderr)
        sys.exit(3)


def ranks_or_relaunch(args) -> int | None:
    """--gpus N means N ranks, one per GPU.  Under torchrun WORLD_SIZE must be
    N (else exit 2).  Started without torchrun and N > 1, bench.py starts the N
    ranks itself through torch.distributed.run (rendezvous on 127.0.0.1) and
    returns that run's exit status; None: carry on in this process."""
    env_world = os.environ.get("WORLD_SIZE")
    if env_world is not None:
        if int(env_world) != args.gpus:
            print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={env_world}: run one rank per GPU", file=sys.stderr)
            return 2
        return None
    if args.gpus <= 1:
        return None
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse_args()
    rc = ranks_or_relaunch(args)
    if rc is not None:
        sys.exit(rc)
    if args.impl == "reference":
        run_reference(args)
    elif args.grid_only:
        import torch

        dev = torch.device("cuda", 0)
        flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
        print(json.dumps(bench_grid_surfaces(args, dev, flush, torch.cuda.current_stream())), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
