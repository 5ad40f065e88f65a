"""CPU: bench.py's multi-rank host logic and its reference arm.

The timing contract takes the max over ranks of every device time; with
N > 1 ranks each rank runs an independent replica. These tests run the
reduction over a world of two gloo ranks on 127.0.0.1, and the reference arm
(the oracle port of the reference's host GROUP BY) as rank 0 and as rank 1.
"""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        got = bench.reduce_max(dist, 1.5 + 2.0 * rank, "cpu")
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 3.5, 1: 3.5}


def test_reduce_max_without_process_group_is_identity():
    sys.path.insert(0, str(REPO))
    import bench

    assert bench.reduce_max(None, 2.25, "cpu") == 2.25


def _reference_arm(rank: int) -> subprocess.CompletedProcess:
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--steps", "3", "--warmup", "3",
           "--rows", "20000"]
    return subprocess.run(cmd, cwd=REPO, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_rank0_prints_one_line():
    r = _reference_arm(0)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "rows/s"
    assert d["cpu_baseline"]["cores"] >= 1 and d["e2e"]["h2d_bytes_per_step"] == 0
    # the reference arm times the whole configured workload every step
    assert d["config"]["rows_per_step"] == 20000 and d["config"]["rows"] == 20000


def test_reference_arm_other_ranks_exit_quietly():
    r = _reference_arm(1)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
