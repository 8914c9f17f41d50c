"""Ensemble sharding across ranks (one process per GPU).

Instances are independent, so an ensemble splits across ranks with no data-path collective:
longest-processing-time-first assignment of instance costs (cells per step) to the currently
lightest rank. Every rank computes the same assignment from the same costs, so no exchange is
needed to agree on it; results are gathered only if the caller wants them on one rank.
"""

from __future__ import annotations

import heapq
from typing import Sequence


def lpt_shards(costs: Sequence[float], n_ranks: int) -> list[list[int]]:
    """Instance indices per rank (each list ascending). Deterministic: ties go to the lower rank."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    heapq.heapify(heap)
    shards: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def shard_loads(costs: Sequence[float], shards: list[list[int]]) -> list[float]:
    return [float(sum(costs[i] for i in s)) for s in shards]
