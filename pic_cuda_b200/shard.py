"""Replicas and job sharding over ranks (one process per GPU).

A single simulation does not shard without a halo exchange per smoothing sweep, so a plain run
at N GPUs is N independent replicas; batched and served jobs are independent, so they are
split over the ranks by work.  Nothing here exchanges simulation data: the only collectives are
the timing and counter reductions of the benchmark (max of the timed region, sum of the work),
which run over whatever process group the caller set up (NCCL on GPUs, gloo on CPU tests).
"""
from __future__ import annotations

import heapq
from typing import Sequence


def shard_jobs(work: Sequence[float], world: int) -> list[list[int]]:
    """Split jobs over `world` ranks by their work (particle-steps): largest first onto the
    least-loaded rank (LPT), ties to the lower rank, so every rank computes the same split
    without communicating.  Returns each rank's job indices in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for j in sorted(range(len(work)), key=lambda k: (-float(work[k]), k)):
        load, r = heapq.heappop(heap)
        out[r].append(j)
        heapq.heappush(heap, (load + float(work[j]), r))
    return [sorted(o) for o in out]


def shard_requests(arrivals: Sequence[float], world: int, rank: int) -> list[int]:
    """The requests rank `rank` serves: every world-th one in arrival order (ties by index), so
    each rank sees a Poisson stream at 1/world of the rate.  Returns indices in arrival order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(arrivals)), key=lambda k: (float(arrivals[k]), k))
    return order[rank::world]


def gather_latencies(lat: Sequence[float], dist=None) -> list[float]:
    """Every rank's request latencies, concatenated in rank order (one rank: a copy)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(x) for x in lat]
    out: list = [None] * dist.get_world_size()
    dist.all_gather_object(out, [float(x) for x in lat])
    return [x for part in out for x in part]


def reduce_timing(ms: float, work: float, dist=None, device=None) -> tuple[float, float]:
    """(max over ranks of the timed region in ms, sum over ranks of the work).  Without a
    process group (one rank) the inputs come back unchanged."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms), float(work)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    w = torch.tensor([float(work)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
