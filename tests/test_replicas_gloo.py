"""The multi-rank (replicas) timing logic of bench.py on two CPU ranks (gloo):
every rank gets the slowest rank's time and the whole-job throughput counts
all replicas.  The GPU path calls the same functions with the NCCL group."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(100.0 + 50.0 * rank, world, "cpu")
        value = bench.replica_throughput(1000, 10, world, ms)
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_throughput_two_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, value in got:
        assert ms == 150.0
        assert value == pytest.approx(1000 * 10 * 2 / 0.150)


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
    assert bench.replica_throughput(10, 2, 1, 1000.0) == 20.0
