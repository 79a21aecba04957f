"""Sharding of independent systems over GPUs (one process per GPU).

A batch of independent systems (the c3 workload) needs no exchange between
GPUs: each rank evaluates its own share, and only the timing is reduced.  The
share is a greedy longest-processing-time partition of an estimated cost per
system (atoms for the pair work, grid points for the PME work), computed the
same way on every rank, so no communication is needed to agree on it.
"""
from __future__ import annotations

import heapq


def system_cost(natoms, grid):
    """Relative cost of one evaluation: pair work ~ atoms, PME ~ grid points."""
    g = int(grid[0]) * int(grid[1]) * int(grid[2])
    return float(natoms) + 0.25 * g


def partition(costs, nranks):
    """Greedy LPT: systems sorted by decreasing cost, each to the least loaded
    rank (ties to the lower rank).  Returns per-rank lists of system indices,
    each in increasing order."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(nranks)]
    out = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(x) for x in out]


def imbalance(costs, parts):
    """max rank load / mean rank load."""
    loads = [sum(costs[i] for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def max_over_ranks(value, device=None):
    """The largest of one float over all ranks of the default process group
    (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
