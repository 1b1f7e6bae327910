"""Independent problems spread over GPUs, one process per GPU.

A single solve does not shard, but a batch of independent problems does: each
rank solves its own share, with no collective on the data path; only the
timing (max over ranks) and the per-problem summaries cross ranks.  Shares are
balanced by the device memory each problem's hierarchy takes, which also
tracks its work (both scale with the cell count).
"""
from __future__ import annotations

from typing import List, Sequence


def estimated_bytes(nx: int, ny: int, mixed: bool = False) -> int:
    """Device bytes of one resident hierarchy (the estimate the solve server
    admits requests by): ~21 FP64 fields per cell over all levels, ~14 FP32
    ones with MGP_FLAG_MIXED, plus fixed buffers."""
    per = 8.0 * 21.0 + (4.0 * 14.0 if mixed else 0.0)
    return int(nx * ny * per) + (8 << 20)


def assign(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time-first: problems by decreasing cost, each to the
    rank with the least load so far (the lowest rank on ties).  Deterministic,
    so every rank computes the same partition without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += costs[k]
    for p in parts:
        p.sort()
    return parts


def my_share(costs: Sequence[float], rank: int, world: int) -> List[int]:
    return assign(costs, world)[rank]


def imbalance(costs: Sequence[float], world: int) -> float:
    """max rank load / mean rank load of the partition."""
    parts = assign(costs, world)
    loads = [sum(costs[k] for k in p) for p in parts]
    mean = sum(loads) / world
    return max(loads) / mean if mean > 0 else 1.0
