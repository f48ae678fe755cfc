"""The bench's multi-rank host logic on CPU (gloo, two ranks).

The Brownian step does not shard: with N GPUs every rank advances its own
replica (seeded 1000 + rank) and the bench reports the whole job's
bead-steps over the slowest rank's device time.  These are the only
collectives on that path, run here as two gloo processes on 127.0.0.1:

* ranks_max: the element-wise maximum of the ranks' (step, e2e) times;
* rank0_choice: rank 0's autotuned cutoff and its timings on every rank;
* without a process group both return their input.
"""
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


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.ranks_max([10.0 + rank, 5.0 - rank], dist)
        picks = bench.rank0_choice([13.6, {"13.6": 1.68}] if rank == 0 else [None, None], dist)
        out[rank] = (t, picks)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_rank0_choice():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        t, picks = res[rank]
        assert t == [11.0, 5.0]
        assert picks == [13.6, {"13.6": 1.68}]


def test_without_process_group():
    import bench
    assert bench.ranks_max([1, 2.5], None) == [1.0, 2.5]
    assert bench.rank0_choice([12.1, None], None) == [12.1, None]
