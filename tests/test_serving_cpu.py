"""CPU: the host side of the sustained serving benchmark (ope_b200.serving:
run_sustained, summarize_sustained) against a fake server -- Poisson
submission, separate reprice and calibration collectors, bounded waits, the
drain deadline with cancellation of what never finishes, and the steady-state
statistics."""
import threading
import time

import numpy as np

from ope_b200 import serving as SV
from ope_b200._lib import OpeError


class FakeServer:
    """Requests finish at once with a latency of 0.1 ms (reprice) or 5 ms
    (calibration); ids in `stuck` never finish until cancelled."""

    def __init__(self, stuck=()):
        self.next = 1
        self.kind = {}
        self.stuck = set(stuck)
        self.cancelled = set()
        self.lock = threading.Lock()

    def _submit(self, kind):
        with self.lock:
            rid = self.next
            self.next += 1
            self.kind[rid] = kind
        return rid

    def submit_price(self, model, contracts, params):
        return self._submit(0)

    def submit_calibrate(self, model, quotes, iv, p0):
        return self._submit(1)

    def wait(self, rid, timeout_ms=-1.0):
        if rid in self.cancelled:
            raise OpeError(7, "cancelled")
        if rid in self.stuck:
            time.sleep(min(max(timeout_ms, 0.0), 5.0) * 1e-3)
            raise OpeError(5, "timeout")
        return None, (0.1 if self.kind[rid] == 0 else 5.0)

    def cancel(self, rid):
        self.cancelled.add(rid)


def _pool():
    con = np.zeros(30, SV.CONTRACT_DTYPE)
    return ([SV.StreamRequest(0, con, np.zeros(8), None, 30)] * 3 +
            [SV.StreamRequest(1, con, np.zeros(5), np.zeros(30), 30)])


def test_sustained_stream_counts_and_cancels_what_never_finishes():
    srv = FakeServer(stuck={3, 10})
    t0 = time.perf_counter()
    res = SV.run_sustained(srv, _pool(), rate=2000.0, seconds=0.25, seed=3, drain_s=0.2)
    assert time.perf_counter() - t0 < 5.0
    n = len(res["latency_ms"])
    assert n == 500 and res["unfinished"] == 2 and not res["errors"]
    assert np.isnan(res["latency_ms"][[2, 9]]).all()  # ids 3 and 10 are submissions 2 and 9
    assert np.isfinite(np.delete(res["latency_ms"], [2, 9])).all()
    assert srv.cancelled == {3, 10}
    row = SV.summarize_sustained(res)
    assert row["requests"] == 500 and row["unfinished_after_drain"] == 2
    assert 0.1 < (row["calibrations_completed_per_s"] / (row["reprices_completed_per_s"] + 1e-9)) < 0.5
    assert row["reprice"]["p50_ms"] == 0.1 and row["calibration"]["p50_ms"] == 5.0
    stuck_kinds = res["kind"][[2, 9]]
    assert row["reprice_sustained"] == (not (stuck_kinds == 0).any())


def test_summary_flags_a_growing_reprice_queue():
    n = 400
    ts = np.linspace(0.0, 10.0, n, endpoint=False)
    res = {"latency_ms": 0.1 + ts, "kind": np.zeros(n, int), "size": np.full(n, 100), "t_submit": ts,
           "offered_rate": 40.0, "arrival_s": 10.0, "wall_s": 12.0, "unfinished": 0, "errors": []}
    row = SV.summarize_sustained(res)
    assert row["reprice_latency_growth"] > 2.0 and not row["reprice_sustained"]
    res["latency_ms"] = np.full(n, 0.2)
    row = SV.summarize_sustained(res)
    assert row["reprice_latency_growth"] == 1.0 and row["reprice_sustained"]
    assert row["reprice_by_size"]["100-499"]["n"] == 200  # the steady half of the submissions
