"""The multi-GPU path of bench.py is replicas only: every rank solves its own
copy and the job time is the max over ranks.  The rank coordination is
checked here with two gloo processes on the CPU."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.replica_barrier(dist)
        out[rank] = bench.replica_max(1.5 + rank, dist, torch.device("cpu"))
        bench.replica_barrier(dist)
    finally:
        dist.destroy_process_group()


def test_replica_max_over_two_gloo_ranks():
    world = 2
    port = 29500 + os.getpid() % 2000
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 2.5


def test_replica_max_without_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_max(3.25, None) == 3.25


def test_reference_arm_rank_nonzero_exits_without_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        m, steps, warmup, gpus = 64, 1, 1, 2
    assert bench.impl_reference(A()) is None
