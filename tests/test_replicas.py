"""Replica mode across ranks (the multi-GPU path: no data-path collective),
run as two gloo processes on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from zldsp_fft_b200 import replicas


def test_shard_covers_every_item_once():
    for n in (0, 1, 7, 20000):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, world) for r in range(world)]
            flat = [i for p in parts for i in p]
            assert flat == list(range(n))
            assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        replicas.shard(10, 2, 2)


def test_aggregate_gbs():
    assert replicas.aggregate_gbs(4e9, 2, 1.0) == 8.0
    with pytest.raises(ValueError):
        replicas.aggregate_gbs(1.0, 1, 0.0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank "times" its replica; the slowest rank sets the job time
        elapsed = 1.0 + rank
        t = replicas.max_over_ranks(elapsed, dist)
        mine = replicas.shard(20000, rank, world)
        out[rank] = (t, replicas.aggregate_gbs(2.0e9, world, t), mine.start, mine.stop)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0
    assert res[0][1] == pytest.approx(2.0)  # 2 ranks x 2 GB / 2 s
    assert (res[0][2], res[0][3], res[1][2], res[1][3]) == (0, 10000, 10000, 20000)
    assert replicas.max_over_ranks(3.5) == 3.5  # no process group: the value itself
