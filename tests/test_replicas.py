"""The multi-GPU form of bench.py is replicas only: one independent domain per
rank, no data-path collective.  Its host logic -- the maximum of the ranks'
device times and the whole-job throughput over it -- runs here on CPU in two
gloo ranks."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r timed 100 + 10 r ms for its replica; the job is as slow as the slowest
        slowest = bench._max_over_ranks(100.0 + 10.0 * rank, world)
        out[rank] = (slowest, bench._aggregate(1000000, 10, world, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replica_timing_is_the_max_over_ranks(world):
    out = mp.get_context("spawn").Manager().dict()  # (no fork: the parent may hold a CUDA context)
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    slowest = 100.0 + 10.0 * (world - 1)
    for r in range(world):
        assert out[r][0] == slowest
        # world x 1e6 cells x 10 steps over the slowest rank's time, in Mcell-steps/s
        assert abs(out[r][1] - world * 1e6 * 10 / (slowest * 1e-3) / 1e6) < 1e-9


def test_single_rank_needs_no_process_group():
    assert bench._max_over_ranks(42.0, 1) == 42.0
    assert bench._aggregate(1000, 2, 1, 1.0) == 1000 * 2 / 1e-3 / 1e6
