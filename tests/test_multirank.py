"""The multi-GPU form of bench.py is N independent replicas (unique quartets are independent; there is
no data-path collective).  What crosses ranks is the timing: every rank reports its own build time and
the job's time is the slowest rank's.  These CPU tests run that reduction with two gloo ranks."""
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


def _rank_main(rank, world, port, results):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, local, w = bench.env_rank()
        own = 10.0 + 5.0 * rank  # this rank's step time (ms)
        results[rank] = (r, local, w, bench.max_over_ranks(own, dist, "cpu"))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        results = m.dict()
        mp.start_processes(_rank_main, args=(world, port, results), nprocs=world, start_method="spawn", join=True)
        res = dict(results)
    assert sorted(res) == [0, 1]
    for rank, (r, local, w, t) in res.items():
        assert (r, local, w) == (rank, rank, world)
        assert t == pytest.approx(15.0)  # the slowest rank's time, on every rank


def test_max_over_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
