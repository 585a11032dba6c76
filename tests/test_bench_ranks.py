"""bench.py's multi-rank arithmetic on two gloo ranks on the CPU: every rank gets the slowest
rank's time, and the job's rate counts every rank's replica over that time."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, device="cpu")
        out[rank] = (ms, bench.job_rate(1000, 20, world, ms))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_take_the_slowest_time():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        got = dict(out)
    for rank in range(world):
        ms, rate = got[rank]
        assert ms == 15.0
        assert rate == pytest.approx(world * 1000 * 20 / 0.015 / 1e6)


def test_one_rank_keeps_its_own_time():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, device="cpu") == 3.5
    assert bench.job_rate(10, 4, 1, 2.0) == pytest.approx(10 * 4 / 0.002 / 1e6)
