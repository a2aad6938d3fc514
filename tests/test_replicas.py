"""Several ranks, as bench.py runs them under torchrun, exercised with the
gloo backend on CPU (world size 2): solves are split with no overlap and no
gap, and the job's time is the slowest rank's."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from gpue_b200 import replicas


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, n, out):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = replicas.shard(n, world, rank)
        got = [None] * world
        dist.all_gather_object(got, mine)
        slowest = replicas.max_over_ranks(1.0 + rank, dist)
        rate, units, secs = replicas.job_rate(100.0 * len(mine), 1.0 + rank, dist)
        out.put((rank, got, slowest, rate, units, secs))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [10, 96, 1])
def test_two_ranks_split_solves_and_take_the_slowest_time(n):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, slowest, rate, units, secs in res:
        flat = sorted(i for part in got for i in part)
        assert flat == list(range(n))                      # every solve once
        assert all(not set(a) & set(b) for a in got for b in got if a is not b)
        assert slowest == 2.0 and secs == 2.0              # max over ranks
        assert units == 100.0 * n and rate == units / 2.0  # all ranks' work


def test_single_process_needs_no_group():
    assert replicas.shard(5, 1, 0) == [0, 1, 2, 3, 4]
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_rate(10.0, 2.0) == (5.0, 10.0, 2.0)
    with pytest.raises(ValueError):
        replicas.shard(5, 2, 2)
