"""CPU, two gloo ranks: the replica timing of bench.py (max over ranks, whole-job
points/s) and a barrier-separated step, the only cross-rank logic the
multi-GPU path has (independent replicas, no data-path collective)."""

import os
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = 10.0 + 5.0 * rank  # rank 1 is the slow one
        dist.barrier()
        ms, value = bench.aggregate_ranks(local, 1000, world, torch.device("cpu"))
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_max_over_ranks():
    world, port = 2, 29531
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, value in got:
        assert ms == 15.0
        assert value == pytest.approx(2 * 1000 / 0.015)


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    ms, value = bench.aggregate_ranks(20.0, 500, 1, torch.device("cpu"))
    assert ms == 20.0 and value == pytest.approx(500 / 0.02)
