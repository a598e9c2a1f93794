"""Replica runs (bench.py --gpus N): world-size-2 process group on CPU
(gloo) — every rank reports its own time, the job uses the slowest rank's
time and all ranks' work; a single process needs no group."""

import os

import pytest
import torch.multiprocessing as mp

from opendynamo_b200 import replicas


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist = replicas.init("gloo", timeout_s=60)
    try:
        own = 1.0 + rank  # rank r "took" 1 + r seconds
        slowest = replicas.max_over_ranks(own, dist)
        out.put((rank, slowest, replicas.job_throughput(100.0, slowest, world)))
    finally:
        replicas.finish(dist)


def test_two_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.0, 2.0]
    assert [r[2] for r in res] == [100.0, 100.0]  # 2 ranks x 100 units / 2 s


def test_single_process_needs_no_group(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "1")
    assert replicas.init("gloo") is None
    assert replicas.max_over_ranks(3.5, None) == 3.5
    assert replicas.world()[0] == 1
