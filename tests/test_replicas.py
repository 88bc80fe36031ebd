"""bench.py's multi-GPU path on the CPU: N replicas over a gloo process
group (world size 2).  The evaluator does not shard within a mesh, so
--gpus N runs N independent replicas; the whole job's time is the slowest
rank's, and its throughput counts every rank's units."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = [10.0 + rank, 20.0 - rank, 1.5 * (rank + 1), 3.0]
        got = bench.replica_max(mine, dist, "cpu")
        q.put((rank, got, bench.replica_rate(world, 30 * 20, got[0] / 1000.0)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_max_over_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, rate in res:
        assert got == [11.0, 20.0, 3.0, 3.0]              # max over the two ranks, same on both
        assert rate == pytest.approx(2 * 600 / 0.011)


def test_single_process_is_identity():
    assert bench.replica_max([1, 2.5], None, "cpu") == [1.0, 2.5]
    assert bench.replica_rate(1, 600, 0.2) == pytest.approx(3000.0)
