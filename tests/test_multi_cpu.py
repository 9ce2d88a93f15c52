"""CPU: the N > 1 path (replicas / weak scaling) with world_size-2 gloo ranks,
and the reference arm's rank handling under torchrun."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "options-pricing-engine-rs_b200")]
    from ope_b200 import multi
    from ope_b200 import workloads as W

    dist = multi.init("gloo", timeout_s=60)
    r, lr, ws = multi.rank_info()
    w = W.c3(n=4096, per_surface=256, seed=multi.shard_seed(3, r))
    multi.barrier(dist)
    elapsed = 1.0 + r  # a stand-in for each rank's timed region
    worst = multi.max_over_ranks(dist, elapsed)
    value = multi.weak_scaling_value(ws, w.n, 5, worst)
    q.put((r, ws, float(w.contracts["strike"][:8].sum()), worst, value))
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_take_the_slowest():
    import random

    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ws0, k0, worst0, v0), (r1, ws1, k1, worst1, v1) = out
    assert (r0, r1) == (0, 1) and ws0 == ws1 == 2
    assert k0 != k1                      # each rank prices its own shard
    assert worst0 == worst1 == 2.0       # max over ranks
    assert v0 == v1 == 2 * 4096 * 5 / 2.0


def test_reference_arm_nonzero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--gpus", "2"], capture_output=True, text=True, env=env, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_reference_arm_prints_one_json_line():
    import json

    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--contracts", "8192", "--cpu-seconds", "0.3"], capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "contracts/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


def test_gpus_flag_must_match_world_size():
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="3")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--gpus", "2"], capture_output=True, text=True, env=env, timeout=120)
    assert p.returncode == 2 and "WORLD_SIZE=3" in p.stderr and p.stdout.strip() == ""


def test_gpus_flag_starts_the_ranks_itself():
    """--gpus 2 without torchrun: bench.py launches two ranks (torch.distributed.run);
    the reference arm's rank 0 prints one line for the 2-rank job, rank 1 nothing."""
    import json

    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR",
                                                          "MASTER_PORT")}
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--gpus", "2", "--contracts", "4096", "--cpu-seconds", "0.2"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["n_gpus"] == 2
