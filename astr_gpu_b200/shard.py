"""Placement of independent boxes on ranks for ensemble runs on several GPUs.

Boxes never exchange data, so a multi-GPU ensemble needs no collective on the data path: each
rank advances its own subset. Subsets come from the longest-processing-time rule (boxes by
decreasing cost, each to the rank with the least cost so far), cost = grid points per step, which
keeps the slowest rank within 4/3 of the optimum."""
from __future__ import annotations

import heapq


def lpt_partition(costs, nparts: int) -> list[list[int]]:
    """Box indices per part, each part's list in increasing index order. Ties go to the lower
    part index, so every rank computes the same placement without communicating."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, p) for p in range(nparts)]
    parts: list[list[int]] = [[] for _ in range(nparts)]
    for i in order:
        load, p = heapq.heappop(heap)
        parts[p].append(i)
        heapq.heappush(heap, (load + costs[i], p))
    return [sorted(x) for x in parts]


def box_cost(n: int) -> int:
    """Grid points of a periodic box with nodes 0..n per axis."""
    return (n + 1) ** 3
