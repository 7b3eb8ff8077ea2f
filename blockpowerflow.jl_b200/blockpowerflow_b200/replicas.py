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


def batch_system_cost(n: int, p: int, qmax: int = 32) -> float:
    """Cost model of one system of a batched solve (the plan's own unit estimate): p columns
    in ceil(p / qmax) slices of width q, each ~1.5 (n / q)^0.7 iterations whose basis traffic
    grows like iterations^2 n q."""
    ns = max(1, -(-int(p) // int(qmax)))
    cost = 0.0
    for k in range(ns):
        q = p // ns + (1 if k < p % ns else 0)
        it = 1.5 * (float(n) / q) ** 0.7
        cost += it * it * float(n) * q
    return cost


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


def allreduce_max(value: float, group=None, device=None) -> float:
    """Max of a scalar over the ranks (the value itself without a process group)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_to_root(local: dict, group=None):
    """Every rank's {system index: result} merged on rank 0 (None on the other ranks): the one
    gather at the end of a sharded batch.  Without a process group, the local dict itself."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return dict(local)
    world = dist.get_world_size(group)
    out = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(local, out, dst=0, group=group)
    if out is None:
        return None
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"system {k} solved on two ranks")
            merged[k] = v
    return merged


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
