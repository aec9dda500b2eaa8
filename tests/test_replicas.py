"""Replicas across ranks (the bench's multi-GPU form): world-size-2 process
groups over gloo on the CPU, the max-over-ranks timing and the whole-job rate,
and the reference arm's ranks above 0 exiting without work."""

import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as td

    w, r, _ = bench.dist_setup(world, backend="gloo")
    # each rank "timed" a different duration; every rank sees the slowest
    ms = bench.max_over_ranks(100.0 + 50.0 * r, w, None)
    bench.barrier(w, None)
    rate = bench.whole_job_rate(w, 1000, ms / 1000.0)
    td.destroy_process_group()
    q.put((r, w, ms, rate))


def test_max_over_ranks_and_whole_job_rate_gloo():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    for _, w, ms, rate in out:
        assert w == 2 and ms == 150.0
        assert rate == pytest.approx(2 * 1000 / 0.15)


def test_reference_arm_rank_above_zero_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
