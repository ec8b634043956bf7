"""The N > 1 host path of bench.py (replicas: one process per GPU, no collective in the data
path) on CPU with two gloo ranks: each rank reports its own device time, the job time is the
slowest rank's, and the whole-job throughput counts every rank's units."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank 0 is slower in the first quantity, rank 1 in the second
        t = bench.max_over_ranks(dist, [100.0 + 50.0 * (rank == 0), 80.0 + 40.0 * (rank == 1)], "cpu")
        dist.barrier()
        q.put((rank, t, bench.replica_throughput(10, world, t[0])))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, thr in out:
        assert t == [150.0, 120.0]
        assert thr == pytest.approx(10 * 2 / 0.150)


def test_single_process_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, [3, 4], "cpu") == [3.0, 4.0]
    assert bench.replica_throughput(5, 1, 500.0) == pytest.approx(10.0)
