"""The bench's multi-rank host logic on two CPU ranks (gloo): the maximum
over ranks of the device time, the whole-job aggregate, and a rank that
fails between steps ending the others' next collective with an error
within the process group's timeout instead of hanging them.  (One GPU per
gpurun call here: the NCCL form of the same calls runs in the driver's
multi-GPU bench.)"""
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _max_worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        # rank r took 10 + 5 r ms: every rank sees the slowest
        m = bench._max_over_ranks(10.0 + 5.0 * rank, world)
        agg = bench._aggregate(64 ** 3, 20, world, m)
        q.put((rank, m, agg))
    finally:
        dist.destroy_process_group()


def _failing_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=5))
    t = torch.ones(1)
    dist.all_reduce(t)  # step 1: both ranks
    if 1 == rank:
        os._exit(3)  # rank 1 fails between steps, with no collective in flight
    try:
        dist.all_reduce(t)  # step 2: rank 0 alone
        q.put((rank, "completed"))
    except Exception as e:  # the timeout or the peer's closed connection
        q.put((rank, "error: " + type(e).__name__))


def _run(target, world=2, timeout=120):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    out = []
    while not q.empty():
        out.append(q.get())
    return out, alive, [p.exitcode for p in procs]


def test_max_over_ranks_and_aggregate_two_ranks():
    out, alive, codes = _run(_max_worker)
    assert not alive, "a rank hung"
    assert sorted(r for r, _, _ in out) == [0, 1], out
    for _, m, agg in out:
        assert m == 15.0
        assert agg == pytest.approx(2 * 64 ** 3 * 20 / 15e-3 / 1e6)


def test_a_failed_rank_ends_the_others_collective():
    out, alive, codes = _run(_failing_worker, timeout=60)
    assert not alive, "a surviving rank hung in its collective"
    res = dict(out)
    assert codes[1] == 3, codes
    assert res.get(0, "").startswith("error"), res
