"""The multi-GPU path of bench.py (replicas of the flow step, one process per GPU) on CPU: two
gloo ranks reduce their step times to the slowest rank's, and the whole-job throughput counts
every replica's updates over that time."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, times, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(torch, times[rank], world, "cpu")
        out[rank] = ms
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("times", [[12.5, 31.0], [40.0, 7.25]])
def test_two_gloo_ranks_take_the_slowest_time(times):
    world = 2
    out = mp.Manager().dict()
    mp.spawn(rank_main, args=(world, free_port(), times, out), nprocs=world, join=True)
    assert out[0] == out[1] == max(times)


def test_replica_throughput_counts_every_replica():
    sys.path.insert(0, ROOT)
    import bench

    one = bench.replica_throughput(1_486_272, 4000, 264.0, 1)
    assert bench.replica_throughput(1_486_272, 4000, 264.0, 4) == pytest.approx(4 * one)
    assert bench.max_over_ranks(torch, 3.5, 1, "cpu") == 3.5
