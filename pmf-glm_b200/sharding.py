"""Placement of independent boxes on ranks for the batched form on several GPUs.

Boxes share nothing during a step, so a multi-GPU batched run is one batch per rank with no
collective in the step: only the placement and a final gather of scalar diagnostics (and the
max-over-ranks time) cross ranks. Placement is longest-processing-time-first: boxes sorted by
cost (N^3 x steps) descending, each given to the least-loaded rank (ties: lower rank; equal
costs keep their input order), which keeps the heaviest rank within 4/3 of the optimum.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def lpt_shard(costs: Sequence[float], world: int) -> List[List[int]]:
    """Box indices per rank (each list in ascending index order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(x) for x in out]


def shard_loads(costs: Sequence[float], shards: Sequence[Sequence[int]]) -> List[float]:
    return [float(sum(costs[i] for i in s)) for s in shards]
