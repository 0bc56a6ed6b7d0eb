"""Multi-GPU sharding of independent planning problems.

Problems never exchange data, so ranks (one process per GPU) take disjoint sets
and run their own persistent launches; the only communication is a barrier and
the reduction of timing / counts.  Nothing on the data path is collective.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_partition(costs, world: int) -> list[np.ndarray]:
    """Longest-processing-time partition: problem indices per rank, largest cost
    first onto the least-loaded rank; every index appears exactly once."""
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(i))
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [np.asarray(sorted(p), dtype=np.int64) for p in parts]


def weak_scaling_seeds(n: int, rank: int, base: int = 100000) -> list[int]:
    """Seeds of the n problems rank `rank` solves when every rank has its own batch."""
    return [base * (rank + 1) + i for i in range(n)]


def reduce_timing(seconds: float, solved: int, device=None):
    """(max seconds over ranks, total solved over ranks); identity without a process group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds), int(solved)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    c = torch.tensor([float(solved)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(round(c.item()))
