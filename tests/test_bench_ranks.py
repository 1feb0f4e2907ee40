"""The multi-GPU bench path is replicas only: each rank times its own steps and the job
rate uses the maximum time over ranks.  Checked here with world_size 2 on the gloo
backend (CPU), as the bench does with NCCL."""

import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        elapsed = [0.5, 0.8][rank]
        el, rate = bench.replica_rate(elapsed, 10, world, dist, torch.device("cpu"))
        out[rank] = (el, rate)
        # the reference arm: rank 0 alone measures and prints; the others return nothing
        class A:
            cpu_seconds = 0.0
            gpus = world
            steps = 1
            warmup = 3
        if rank != 0:
            assert bench.run_reference(A, rank) is None
    finally:
        dist.destroy_process_group()


def test_replica_rate_two_ranks_gloo():
    world, port = 2, 29517
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        el, rate = out[r]
        assert el == pytest.approx(0.8)
        assert rate == pytest.approx(2 * 10 / 0.8)
