"""Placing many independent block systems on several GPUs.

One system does not shard: after the coloring order its element rows form a strict
elimination chain, so a single system runs on one GPU (other GPUs hold replicas).
Independent systems do shard, with no exchange between GPUs on the data path: each rank
factors and solves the systems assigned to it, and only per-system results (residuals,
iteration counts, timings) are gathered at the end.

The assignment is longest-processing-time first (LPT) on the exact factorization flops
of each system from the host symbolic phase, which bounds the slowest rank at 4/3 of
the optimum.
"""

from __future__ import annotations

import heapq

import numpy as np


def assign_lpt(weights, world_size: int) -> list[list[int]]:
    """Indices of `weights` per rank: heaviest first, each to the least-loaded rank.

    Ties go to the lowest rank, so every rank computes the same assignment.
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    heap = [(0.0, r) for r in range(world_size)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(w[i]), r))
    for r in range(world_size):
        out[r].sort()
    return out


def loads(weights, assignment) -> list[float]:
    w = np.asarray(weights, dtype=np.float64)
    return [float(w[idx].sum()) if idx else 0.0 for idx in assignment]
