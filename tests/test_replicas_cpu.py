"""Multi-GPU plumbing on CPU: the unit split and the cross-rank reductions,
with two gloo ranks (127.0.0.1) standing in for two GPUs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from psgpu_b200.replicas import cost2d, max_over_ranks, shard, sum_over_ranks


def test_shard_covers_every_unit_once_and_balances():
    rng = np.random.default_rng(1)
    sizes = rng.choice([64, 128, 256], 512)
    costs = [cost2d(int(n)) for n in sizes]
    for world in (1, 2, 3, 8):
        parts = shard(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert shard([1.0, 1.0, 1.0], 2) == [[0, 2], [1]]


def test_shard_is_deterministic():
    costs = [3.0, 1.0, 2.0, 2.0, 5.0]
    assert shard(costs, 2) == shard(list(costs), 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [cost2d(n) for n in (64, 256, 128, 128, 64, 256, 32)]
        mine = shard(costs, world)[rank]
        done = sum_over_ranks(len(mine), dist)
        slowest = max_over_ranks(1.0 + rank, dist)
        # every rank sees the same split and the same reductions
        allparts = [None] * world
        dist.all_gather_object(allparts, mine)
        q.put((rank, done, slowest, allparts))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_reduce():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, done, slowest, parts in res:
        assert done == 7
        assert slowest == 2.0
        assert sorted(i for p in parts for i in p) == list(range(7))
