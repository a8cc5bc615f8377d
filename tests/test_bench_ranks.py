"""bench.py's multi-rank aggregation (replicas, one per GPU) on CPU with gloo.

Every rank runs an independent replica; the job time is the slowest rank's
device time (max over ranks) and the throughput counts all ranks' work.  This
runs the same helpers bench.py uses, with two gloo ranks on 127.0.0.1.
"""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 100.0 + 25.0 * rank          # rank 1 is the slow one
        t = bench.max_over_ranks(ms, world, "cpu")
        out[rank] = (t, bench.replica_throughput(1.0e9, t, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_max_time_and_whole_job_throughput():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        t, v = out[r]
        assert t == pytest.approx(125.0)
        assert v == pytest.approx(2 * 1.0e9 / 0.125)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5
    assert bench.replica_throughput(3.0e9, 1500.0, 1) == pytest.approx(2.0e9)
