"""Problem partitioning across GPUs (one process per GPU): the partition is
deterministic, covers every problem once and stays balanced; two gloo ranks
on the CPU compute the same partition and agree on the max-over-ranks time."""
from __future__ import annotations

import os
import socket
from datetime import timedelta

import pytest

from mgpoisson2d_b200 import partition as P
from mgpoisson2d_b200 import workloads as W


def _costs(n=512, mixed=True):
    out = []
    for i in range(n):
        nx, ny, *_ = W.batch_problem_params(i)
        out.append(float(P.estimated_bytes(nx, ny, mixed)))
    return out


def test_partition_covers_every_problem_once_and_balances():
    costs = _costs()
    for world in (1, 2, 4, 8):
        parts = P.assign(costs, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        assert P.imbalance(costs, world) < 1.05
        assert parts == P.assign(costs, world)   # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, costs, q):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        share = P.my_share(costs, rank, world)
        parts = [None] * world
        dist.all_gather_object(parts, share)
        t = torch.tensor([sum(costs[k] for k in share)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, parts, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_partition():
    import multiprocessing as mp
    costs = _costs(96)
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = P.assign(costs, world)
    loads = [sum(costs[k] for k in part) for part in expect]
    for rank, parts, tmax in sorted(out):
        assert parts == expect
        assert tmax == pytest.approx(max(loads))
