"""Replicas (the multi-GPU mode of this path): the bench's aggregation over
ranks, exercised with two gloo processes on CPU.  The path has no exchange
step, so ranks share nothing but the barrier and the max-over-ranks timing."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, values, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        out[rank] = bench.max_over_ranks(values[rank], "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    world = 2
    values = [[1.5, 9.0], [2.5, 3.0]]
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), values, out), nprocs=world, join=True)
        got = dict(out)
    assert got[0] == got[1] == [2.5, 9.0]


def test_replica_value_is_weak_scaling():
    import bench

    assert bench.replica_value(1, 10, 2.0) == 5.0
    assert bench.replica_value(4, 10, 2.5) == pytest.approx(16.0)
