"""CPU, two gloo ranks: the multi-GPU host logic (sharding of independent jobs, whole-job
throughput as all ranks' units over the slowest rank's time)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from b12_b200.ranks import max_over_ranks, shard, sum_over_ranks, throughput
from b12_b200.workloads import job_stream


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        stream = job_stream(101, 500.0, 0)
        mine = shard(stream, world, rank)
        ids = [None] * world
        dist.all_gather_object(ids, [j["id"] for j in mine])
        # every job owned by exactly one rank
        flat = sorted(i for part in ids for i in part)
        units = float(len(mine))
        seconds = 1.0 + rank              # rank 1 is the slow one
        rate, total, slowest = throughput(dist, units, seconds)
        out[rank] = dict(flat=flat, total=total, slowest=slowest, rate=rate,
                         mx=max_over_ranks(dist, 10.0 * rank), sm=sum_over_ranks(dist, 1.0))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_aggregate():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        assert res[r]["flat"] == list(range(101))
        assert res[r]["total"] == 101.0 and res[r]["slowest"] == 2.0
        assert res[r]["rate"] == pytest.approx(50.5)
        assert res[r]["mx"] == 10.0 and res[r]["sm"] == 2.0


def test_shard_without_ranks():
    items = list(range(10))
    assert shard(items, 1, 0) == items
    assert shard(items, 3, 2) == [2, 5, 8]
    with pytest.raises(ValueError):
        shard(items, 2, 2)
    assert max_over_ranks(None, 3.0) == 3.0 and throughput(None, 10.0, 2.0) == (5.0, 10.0, 2.0)
