"""Multi-GPU replicas: one process per GPU, requests sharded across ranks.

The generation path has no exchange step: points, realizations and requests
are independent once the wavevector/phase tables of a request are built, and
those are built per request on its own GPU.  N GPUs therefore run as N
independent replicas (weak scaling for the headline step, request sharding
for batches); the only collectives are the host-side reductions of the
timing: the total work (sum) and the slowest rank's time (max).  Nothing on
the data path crosses NVLink.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def replica_seed(seed_start: int, rank: int) -> int:
    """seed_start of rank `rank`'s replica (distinct rnglib streams)."""
    return int(seed_start) + int(rank)


def shard_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of requests to ranks: the most
    expensive request first, each to the least-loaded rank.  Deterministic
    (ties broken by index), so every rank computes the same plan."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for lst in out:
        lst.sort()
    return out


def aggregate(local_units: float, local_seconds: float, dist=None, device=None):
    """(total units over ranks, slowest rank's seconds): the whole-job
    throughput is total / slowest.  Without an initialised process group the
    local values are returned."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(local_units), float(local_seconds)
    import torch

    t = torch.tensor([float(local_units), float(local_seconds)], dtype=torch.float64, device=device)
    u = t[:1].clone()
    s = t[1:].clone()
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    dist.all_reduce(s, op=dist.ReduceOp.MAX)
    return float(u.item()), float(s.item())
