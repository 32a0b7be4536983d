"""The multi-process path of bench.py on the host: two gloo ranks (one process
each, as torchrun starts them) time the same region for different durations;
every rank gets the slowest rank's time, and the whole-job rate counts every
rank's steps over that time (replicas, weak scaling)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.reduce_max_over_ranks(dist, times[rank], "cpu")
        out[rank] = (ms, bench.job_rate(world, 100, ms))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_count_every_step():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    times = [180.0, 250.5]  # ms of the same timed region on rank 0 and rank 1
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a gloo rank did not finish")
        assert p.exitcode == 0
    for r in range(2):
        ms, rate = out[r]
        assert ms == 250.5
        assert rate == pytest.approx(2 * 100 / 0.2505)


def test_one_process_keeps_its_own_time():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max_over_ranks(None, 123.25, "cpu") == 123.25
    assert bench.job_rate(1, 200, 400.0) == pytest.approx(500.0)
