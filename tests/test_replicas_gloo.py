"""The replica plumbing with two gloo ranks on CPU: max-over-ranks timing,
whole-job throughput and request sharding."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fennol_b200.replicas import job_throughput, max_over_ranks, shard, sum_over_ranks


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        t = [0.25, 0.75][rank]
        units = [1000, 3000][rank]
        items = list(range(11))
        mine = shard(items, rank, world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        out[rank] = {"max": max_over_ranks(t), "sum": sum_over_ranks(units),
                     "rate": job_throughput(units, t), "shards": got}
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_sharding():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    for r in range(world):
        assert res[r]["max"] == 0.75
        assert res[r]["sum"] == 4000
        assert abs(res[r]["rate"] - 4000 / 0.75) < 1e-9
    shards = res[0]["shards"]
    assert sorted(sum(shards, [])) == list(range(11))
    assert not set(shards[0]) & set(shards[1])


def test_single_process_fallbacks():
    assert max_over_ranks(2.5) == 2.5 and sum_over_ranks(3) == 3.0
    assert job_throughput(10, 2.0) == 5.0
    assert shard(list("abcde"), 1, 2) == ["b", "d"]
    with pytest.raises(ValueError):
        shard([1], 2, 2)
