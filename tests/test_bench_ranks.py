"""The benchmark's multi-rank plumbing on the CPU (gloo, world size 2).

bench.py runs one process per GPU under torchrun; ranks are independent
replicas of the workload (no data-path collective), joined by a barrier on
both sides of the timed region and a max-reduction of the per-rank device
times. These tests run that plumbing with the gloo backend on two CPU ranks.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local = bench.dist_env()
    assert (w, r, local) == (world, rank, rank)
    dist = bench.init_dist(w, "gloo")
    bench.barrier(dist)
    # Each rank's device time differs; every rank must see the slowest one.
    slowest = bench.reduce_max(dist, 10.0 + 3.5 * rank, "cpu")
    bench.barrier(dist)
    results[rank] = slowest
    dist.destroy_process_group()


def test_ranks_agree_on_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    results = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, results))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(results) == {0: 13.5, 1: 13.5}


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.init_dist(1, "gloo") is None
    assert bench.reduce_max(None, 4.25, "cpu") == 4.25
    bench.barrier(None)


def test_reference_arm_prints_one_line_under_torchrun():
    sys.path.insert(0, ROOT)
    import oracle

    if not oracle.Reference.available():
        pytest.skip("the reference library has not been built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--workload",
           "direct-plummer-4096"]
    out = subprocess.run(["timeout", "-k", "10", "300"] + cmd, cwd=ROOT, capture_output=True,
                         text=True, env={**os.environ, "OMP_NUM_THREADS": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
