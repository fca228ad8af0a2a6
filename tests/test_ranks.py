"""The N > 1 host path of bench.py on CPU: two gloo ranks (replicas only).

Each rank times its own replica; the job's time is the slowest rank's (one
MAX all-reduce that every rank takes) and its throughput is the units all
ranks processed over that time.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT  # noqa: F401  (puts the repository on sys.path)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = 100.0 + 25.0 * rank           # this rank's replica time, ms
        slowest = bench.max_over_ranks(mine, "cpu")
        dist.barrier()
        results[rank] = (slowest, bench.job_rate(4096 * 3, world, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_sum_the_work():
    world = 2
    with mp.Manager() as manager:
        results = manager.dict()
        mp.start_processes(_rank, args=(world, _free_port(), results), nprocs=world,
                           start_method="spawn", join=True)
        got = dict(results)
    expected_ms = 125.0
    for rank in range(world):
        slowest, rate = got[rank]
        assert slowest == expected_ms
        assert rate == pytest.approx(world * 4096 * 3 / (expected_ms / 1e3))


def test_one_rank_keeps_its_own_time():
    import bench
    assert not dist.is_initialized()
    assert bench.max_over_ranks(42.0, "cpu") == 42.0
    assert bench.job_rate(10, 1, 1000.0) == pytest.approx(10.0)


def _failing_rank(rank, world, port, results):
    """Rank 1 leaves between steps (its replica failed), before the timing
    collective; rank 0 must learn it from the closed connection or the short
    process-group timeout, not wait for good."""
    import datetime
    import time
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    try:
        if rank == 1:
            results[rank] = "left"
            return
        t0 = time.monotonic()
        try:
            bench.max_over_ranks(10.0, "cpu")
            results[rank] = "collective completed"
        except Exception as exc:  # gloo reports the missing peer
            results[rank] = ("error", type(exc).__name__, time.monotonic() - t0)
    finally:
        if rank == 0:
            dist.destroy_process_group()


def test_a_failed_rank_ends_the_others_collective_with_an_error():
    world = 2
    with mp.Manager() as manager:
        results = manager.dict()
        ctx = mp.start_processes(_failing_rank, args=(world, _free_port(), results),
                                 nprocs=world, start_method="spawn", join=False)
        deadline = __import__("time").monotonic() + 120
        while not ctx.join(timeout=1):
            if __import__("time").monotonic() > deadline:
                for p in ctx.processes:
                    p.kill()
                pytest.fail("ranks did not end")
        got = dict(results)
    assert got[1] == "left"
    assert got[0][0] == "error" and got[0][2] < 60


def _absent_rank(index, port, results):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=0, world_size=2,
                                timeout=datetime.timedelta(seconds=3))
        results[0] = "joined"
    except Exception as exc:
        results[0] = ("error", type(exc).__name__)


def test_a_rank_that_never_joins_ends_the_rendezvous_with_an_error():
    with mp.Manager() as manager:
        results = manager.dict()
        mp.start_processes(_absent_rank, args=(_free_port(), results), nprocs=1,
                           start_method="spawn", join=True)
        got = dict(results)
    assert got[0][0] == "error"
