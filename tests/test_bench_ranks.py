"""bench.py's multi-rank arithmetic on CPU: two gloo ranks (one process
each, as torchrun launches them) reduce their step times to the slowest
rank's, and the whole-job rate counts every rank's replica."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, loc = bench.dist_setup(None)
        t = bench.reduce_max(times[rank], dist)
        out[rank] = (w, r, loc, t, bench.whole_job_rate(w, 1.0e12, 3, t))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    times = [1500.0, 1750.0]
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, times, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        w, r, loc, t, rate = res[rank]
        assert (w, r, loc) == (world, rank, rank)
        assert t == max(times)
        assert rate == pytest.approx(world * 1.0e12 * 3 / (max(times) * 1e-3))


def test_one_rank_is_its_own_maximum():
    import bench
    assert bench.reduce_max(12.5, None) == 12.5
    assert bench.whole_job_rate(1, 2.0e12, 4, 1000.0) == pytest.approx(8.0e12)
