"""The multi-GPU form of the benchmark is replicas only: every rank searches its own copy of the
workload and the job's time is the slowest rank's. This checks, on the CPU with two gloo ranks,
the reduction bench.py uses for that (element-wise maximum over ranks) and the whole-job
throughput it reports."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = [10.0 + 5.0 * rank, 20.0 - 3.0 * rank]  # per-rank step and end-to-end ms
        got = bench.reduce_max(mine, dist, "cpu")
        out.put((rank, got, bench.replica_throughput(1_000_000, world, got[0])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replica_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, value in res:
        assert got == [15.0, 20.0]  # max over ranks of each value
        assert value == pytest.approx(2 * 1_000_000 / 0.015)


def test_single_process_reduction_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_max([1.5, 2.5], None, "cpu") == [1.5, 2.5]
    assert bench.replica_throughput(100, 1, 10.0) == pytest.approx(10_000.0)
