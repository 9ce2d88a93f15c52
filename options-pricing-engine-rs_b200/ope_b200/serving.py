"""Python handle on the device-resident request server (include/ope.h
ope_server_*) and a Poisson load generator for the serving benchmark.

The server itself is native (csrc/serving.cu): a scheduler thread packs
pending requests into micro-batches, admits them by device memory, runs
several on different streams at once and records per-request latency.
"""
from __future__ import annotations

import ctypes
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import api
from ._lib import MODEL_BATES, MODEL_HESTON, OpeError, check, load
from .workloads import CONTRACT_DTYPE

OPE_ERR_TIMEOUT, OPE_ERR_REJECTED, OPE_ERR_CANCELLED = 5, 6, 7


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("tol", ctypes.c_double),
        ("hbm_fraction", ctypes.c_double),
        ("hbm_cap_bytes", ctypes.c_uint64),
        ("max_inflight", ctypes.c_uint32),
        ("max_batch_contracts", ctypes.c_uint32),
        ("pinned_bytes", ctypes.c_uint64),
        ("calib_sm_fraction", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in (
        "submitted", "completed", "rejected", "cancelled", "failed", "batches", "batched_requests", "max_inflight",
        "hbm_budget_bytes", "hbm_peak_bytes", "pending", "inflight")]


class Server:
    """A running server.  submit_* return request ids; wait() returns (result, latency_ms)."""

    def __init__(self, tol: float = api.REF_TOL, hbm_fraction: float = 0.5, hbm_cap_bytes: int = 0,
                 max_inflight: int = 4, max_batch_contracts: int = 0, pinned_bytes: int = 0,
                 calib_sm_fraction: float = 0.5):
        cfg = ServerConfig(tol=tol, hbm_fraction=hbm_fraction, hbm_cap_bytes=hbm_cap_bytes,
                           max_inflight=max_inflight, max_batch_contracts=max_batch_contracts,
                           pinned_bytes=pinned_bytes, calib_sm_fraction=calib_sm_fraction)
        h = ctypes.c_void_p()
        check(load().ope_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._kinds: dict[int, tuple[int, int]] = {}
        self._lock = threading.Lock()

    def close(self) -> None:
        if self._h:
            load().ope_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit_price(self, model: int, contracts, params) -> int:
        con = api.contracts_array(contracts)
        p = np.ascontiguousarray(params, dtype=np.float64)
        rid = ctypes.c_uint64()
        check(load().ope_server_submit_price(self._h, model, con.ctypes.data, con.size, p.ctypes.data,
                                             ctypes.byref(rid)))
        with self._lock:
            self._kinds[rid.value] = (0, con.size)
        return rid.value

    def submit_calibrate(self, model: int, quotes, iv_market, p0) -> int:
        con = api.contracts_array(quotes)
        iv = np.ascontiguousarray(iv_market, dtype=np.float64)
        p = np.ascontiguousarray(p0, dtype=np.float64)
        rid = ctypes.c_uint64()
        check(load().ope_server_submit_calibrate(self._h, model, con.ctypes.data, iv.ctypes.data, con.size,
                                                 p.ctypes.data, ctypes.byref(rid)))
        with self._lock:
            self._kinds[rid.value] = (1, con.size)
        return rid.value

    def wait(self, rid: int, timeout_ms: float = -1.0):
        """Block until request `rid` finishes: (prices | calib record, latency_ms).  Raises OpeError."""
        with self._lock:
            kind, n = self._kinds[rid]
        lat = ctypes.c_double()
        if kind == 0:
            out = np.empty(n)
            rc = load().ope_server_wait(self._h, rid, timeout_ms, out.ctypes.data, None, ctypes.byref(lat))
        else:
            out = np.zeros(1, api.CALIB_RESULT_DTYPE)
            rc = load().ope_server_wait(self._h, rid, timeout_ms, None, out.ctypes.data, ctypes.byref(lat))
            out = out[0]
        if rc != OPE_ERR_TIMEOUT:
            with self._lock:
                self._kinds.pop(rid, None)
        check(rc)
        return out, lat.value

    def cancel(self, rid: int) -> None:
        check(load().ope_server_cancel(self._h, rid))

    def stats(self) -> dict:
        s = ServerStats()
        check(load().ope_server_get_stats(self._h, ctypes.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in s._fields_}


# ------------------------------------------------------------- load generator
@dataclass
class StreamRequest:
    kind: int                  # 0 reprice (Bates), 1 calibration (Heston)
    contracts: np.ndarray
    params: np.ndarray
    iv: np.ndarray | None = None
    size: int = 0


def _surface(rng, n: int, params_h: np.ndarray):
    nt = max(1, int(round(np.sqrt(n / 4))))
    nk = int(np.ceil(n / nt))
    T = np.sort(np.exp(rng.uniform(np.log(1 / 52), np.log(3.0), nt)))
    m = np.sort(rng.uniform(-0.5, 0.4, nk))
    TT, MM = np.meshgrid(T, m, indexing="ij")
    r, q = rng.uniform(0.0, 0.06), rng.uniform(0.0, 0.03)
    con = np.zeros(TT.size, CONTRACT_DTYPE)
    con["spot"], con["strike"] = 100.0, (100.0 * np.exp((r - q) * TT) * np.exp(MM)).ravel()
    con["expiry"], con["rate"], con["div_yield"], con["vol"] = TT.ravel(), r, q, 0.2
    con["opt_type"] = np.where(MM.ravel() >= 0.0, 0, 1)
    return con[:n]


def make_stream(n_requests: int, seed: int = 5, calib_share: float = 0.2, lo: int = 20, hi: int = 2000):
    """Config 5 mix: 80 % Bates surface reprices / 20 % Heston calibrations,
    sizes log-uniform in [lo, hi] contracts, parameters drawn as in config 2
    (plus config 3's jump ranges for Bates).  Calibration market IVs are the
    model IVs of a seeded true parameter set (device pricer + device IV) plus
    N(0, 0.005) noise; start points truth x U(0.7, 1.3)."""
    from .workloads import _heston_draw, feller_heston_draw

    rng = np.random.default_rng(seed)
    out: list[StreamRequest] = []
    for _ in range(n_requests):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        if rng.uniform() < calib_share:
            truth = feller_heston_draw(rng, 1)[0]
            con = _surface(rng, n, truth)
            px = api.batch_heston(con, truth, tol=api.REF_TOL)
            iv, ok = api.batch_implied_vol(con, px)
            ok &= (iv > 0.01) & (iv < 2.0)
            con, iv = con[ok], np.maximum(iv[ok] + rng.normal(0.0, 0.005, int(ok.sum())), 1e-3)
            if con.size == 0:
                continue
            out.append(StreamRequest(1, con, truth * rng.uniform(0.7, 1.3, 5), iv, con.size))
        else:
            h = _heston_draw(rng, 1)[0]
            jp = np.array([rng.uniform(0.0, 1.5), rng.uniform(-0.3, 0.1), rng.uniform(0.05, 0.4)])
            con = _surface(rng, n, h)
            out.append(StreamRequest(0, con, np.concatenate([h, jp]), None, con.size))
    return out


def run_stream(server: Server, reqs: list[StreamRequest], rate: float, seed: int = 7) -> dict:
    """Submit `reqs` at Poisson arrival times (rate req/s) while a collector
    thread waits for completions.  Returns per-request latencies and the
    achieved throughput."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(reqs))
    ids: list[tuple[int, int, int]] = []  # (rid, kind, size)
    lat = np.full(len(reqs), np.nan)
    errors: list[str] = []
    done = threading.Event()
    cond = threading.Condition()

    def collector():
        k = 0
        while k < len(reqs):
            with cond:
                while k >= len(ids):
                    cond.wait(0.01)
                rid, kind, size = ids[k]
            try:
                _, ms = server.wait(rid)
                lat[k] = ms
            except OpeError as e:
                errors.append(str(e))
            k += 1
        done.set()

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    t_next = t0
    for r, g in zip(reqs, gaps):
        t_next += g
        now = time.perf_counter()
        if t_next > now:
            time.sleep(t_next - now)
        if r.kind == 0:
            rid = server.submit_price(MODEL_BATES, r.contracts, r.params)
        else:
            rid = server.submit_calibrate(MODEL_HESTON, r.contracts, r.iv, r.params)
        with cond:
            ids.append((rid, r.kind, r.size))
            cond.notify()
    done.wait()
    t_end = time.perf_counter()
    kinds = np.array([k for _, k, _ in ids])
    sizes = np.array([s for _, _, s in ids])
    return {"latency_ms": lat, "kind": kinds, "size": sizes, "wall_s": t_end - t0, "errors": errors,
            "offered_rate": rate, "achieved_rate": len(reqs) / (t_end - t0)}


def summarize(res: dict) -> dict:
    lat, kinds, sizes = res["latency_ms"], res["kind"], res["size"]
    out = {"offered_req_per_s": res["offered_rate"], "achieved_req_per_s": res["achieved_rate"],
           "requests": int(lat.size), "errors": len(res["errors"]),
           "contracts_per_s": float(sizes[kinds == 0].sum() / res["wall_s"])}
    for name, sel in (("reprice", kinds == 0), ("calibration", kinds == 1)):
        if sel.any():
            out[name] = {"p50_ms": float(np.nanpercentile(lat[sel], 50)), "p99_ms": float(np.nanpercentile(lat[sel], 99)),
                         "n": int(sel.sum())}
    buckets = [(20, 100), (100, 500), (500, 2001)]
    out["reprice_by_size"] = {}
    for lo, hi in buckets:
        sel = (kinds == 0) & (sizes >= lo) & (sizes < hi)
        if sel.any():
            out["reprice_by_size"][f"{lo}-{hi - 1}"] = {
                "p50_ms": float(np.nanpercentile(lat[sel], 50)), "p99_ms": float(np.nanpercentile(lat[sel], 99)),
                "n": int(sel.sum())}
    return out


def run_sustained(server: Server, pool: list[StreamRequest], rate: float, seconds: float, seed: int = 7,
                  calib_share: float = 0.2, drain_s: float = 20.0) -> dict:
    """A fresh Poisson stream at `rate` req/s for `seconds` of arrivals: each
    arrival is a calibration with probability calib_share, else a reprice,
    its contents drawn from `pool` (the server keeps no results between
    requests, so repeated contents cost as much as new ones).  Reprices and
    calibrations are collected by separate threads, so a saturated
    calibration queue never delays the bookkeeping of reprices.  Whatever is
    unfinished `drain_s` after the last arrival is cancelled and counted."""
    rng = np.random.default_rng(seed)
    rep = [r for r in pool if r.kind == 0]
    cal = [r for r in pool if r.kind == 1]
    n = max(1, int(round(rate * seconds)))
    is_cal = (rng.uniform(size=n) < calib_share) if cal else np.zeros(n, bool)
    which = np.where(is_cal, rng.integers(0, max(1, len(cal)), n), rng.integers(0, len(rep), n))
    gaps = rng.exponential(1.0 / rate, n)
    t_sub = np.full(n, np.nan)
    lat = np.full(n, np.nan)
    size = np.array([(cal[w] if c else rep[w]).size for c, w in zip(is_cal, which)])
    queues = {0: [], 1: []}  # per kind: (index, rid) in submission order
    cond = threading.Condition()
    state = {"deadline": None, "unfinished": 0, "errors": []}
    finished = {0: threading.Event(), 1: threading.Event()}

    def collector(kind: int):
        k = 0
        while True:
            with cond:
                while k >= len(queues[kind]) and state["deadline"] is None:
                    cond.wait(0.01)
                if k >= len(queues[kind]):
                    break
                i, rid = queues[kind][k]
            k += 1
            while True:  # bounded waits: the drain deadline is re-read between them
                deadline = state["deadline"]
                timeout = 50.0 if deadline is None else max(0.0, 1e3 * (deadline - time.perf_counter()))
                try:
                    _, ms = server.wait(rid, timeout)
                    lat[i] = ms
                    break
                except OpeError as e:
                    if e.status != OPE_ERR_TIMEOUT:
                        state["errors"].append(str(e))
                        break
                    if deadline is not None and time.perf_counter() >= deadline:
                        server.cancel(rid)
                        try:
                            server.wait(rid, 10000.0)
                        except OpeError:
                            pass
                        with cond:
                            state["unfinished"] += 1
                        break
        finished[kind].set()

    threads = [threading.Thread(target=collector, args=(kd,), daemon=True) for kd in (0, 1)]
    for th in threads:
        th.start()
    t0 = time.perf_counter()
    t_next = t0
    for i in range(n):
        t_next += gaps[i]
        now = time.perf_counter()
        if t_next > now:
            time.sleep(t_next - now)
        r = cal[which[i]] if is_cal[i] else rep[which[i]]
        t_sub[i] = time.perf_counter() - t0
        if r.kind == 0:
            rid = server.submit_price(MODEL_BATES, r.contracts, r.params)
        else:
            rid = server.submit_calibrate(MODEL_HESTON, r.contracts, r.iv, r.params)
        with cond:
            queues[r.kind].append((i, rid))
            cond.notify_all()
    t_arr = time.perf_counter() - t0
    with cond:
        state["deadline"] = time.perf_counter() + drain_s
        cond.notify_all()
    for kd in (0, 1):
        finished[kd].wait()
    return {"latency_ms": lat, "kind": is_cal.astype(int), "size": size, "t_submit": t_sub, "offered_rate": rate,
            "arrival_s": t_arr, "wall_s": time.perf_counter() - t0, "unfinished": state["unfinished"],
            "errors": state["errors"]}


def summarize_sustained(res: dict) -> dict:
    """Per stream: the arrival period, what was submitted and completed per
    second of it, latency percentiles over the steady half (requests
    submitted in the second half of the arrival period), by kind and by
    reprice size, and the growth of the reprice latency across the run (the
    median of the last quarter of submissions over that of the second
    quarter: a queue that keeps growing shows here as a ratio well above 1)."""
    lat, kind, size, ts = res["latency_ms"], res["kind"], res["size"], res["t_submit"]
    T = res["arrival_s"]
    done = np.isfinite(lat)
    rep, cal = kind == 0, kind == 1
    steady = ts >= 0.5 * T
    out = {"offered_req_per_s": res["offered_rate"], "arrival_s": T, "wall_s": res["wall_s"],
           "submitted_req_per_s": float(len(lat) / T), "requests": int(len(lat)),
           "reprices_completed_per_s": float((rep & done).sum() / T),
           "reprice_contracts_per_s": float(size[rep & done].sum() / T),
           "calibrations_completed_per_s": float((cal & done).sum() / T),
           "unfinished_after_drain": int(res["unfinished"]), "errors": len(res["errors"])}
    for name, sel in (("reprice", rep), ("calibration", cal)):
        sel = sel & done & steady
        if sel.any():
            out[name] = {"p50_ms": float(np.percentile(lat[sel], 50)), "p99_ms": float(np.percentile(lat[sel], 99)),
                         "n": int(sel.sum())}
    out["reprice_by_size"] = {}
    for lo, hi in ((20, 100), (100, 500), (500, 2001)):
        sel = rep & done & steady & (size >= lo) & (size < hi)
        if sel.any():
            out["reprice_by_size"][f"{lo}-{hi - 1}"] = {
                "p50_ms": float(np.percentile(lat[sel], 50)), "p99_ms": float(np.percentile(lat[sel], 99)),
                "n": int(sel.sum())}
    q2 = rep & done & (ts >= 0.25 * T) & (ts < 0.5 * T)
    q4 = rep & done & (ts >= 0.75 * T)
    growth = float(np.median(lat[q4]) / np.median(lat[q2])) if q2.any() and q4.any() else None
    out["reprice_latency_growth"] = growth
    out["reprice_sustained"] = bool((rep & ~done).sum() == 0 and growth is not None and growth < 2.0)
    return out
