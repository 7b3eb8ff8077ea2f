"""Multi-GPU: independent systems spread over ranks, no collective on the data path.

A single power-flow system is not partitioned across GPUs (a row split would need a halo
exchange per SpMM and an all-reduce per Gram product).  What shards are independent systems
(grids, Newton steps, right-hand-side groups): `assign_systems` balances them over the ranks by
estimated cost (longest-processing-time-first), each rank solves its own with the single-GPU
library, and `aggregate` combines the per-rank results once at the end (sum of converged
right-hand sides, max of the device times), the only collective.
"""
from __future__ import annotations

import heapq


def solve_cost(n: int, nnz: int, p: int, iters: int = 50) -> float:
    """Cost model of one block-GMRES solve: per iteration the sparse work (SpMM + two
    triangular sweeps, ~3 nnz p) plus the Gram-Schmidt work growing with the basis
    (~8 n p^2 k); summed over `iters` iterations."""
    return iters * 3.0 * nnz * p + 8.0 * n * p * p * iters * (iters + 1) / 2.0


def assign_systems(costs, world: int):
    """Longest-processing-time-first assignment of systems to `world` ranks.

    Returns a list (one per rank) of system indices; deterministic for equal costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for lst in out:
        lst.sort()
    return out


def aggregate(local_rhs: float, local_ms: float, group=None, device=None):
    """(total converged RHS over ranks, max device time over ranks) -- one all-reduce each."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(local_rhs), float(local_ms)
    dev = device if device is not None else "cpu"
    t = torch.tensor([float(local_rhs)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    m = torch.tensor([float(local_ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    return float(t.item()), float(m.item())
