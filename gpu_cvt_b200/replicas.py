"""Multi-GPU: replicas, one process per GPU.

The remesh path shards at mesh granularity -- meshes (or requests) are
independent and a Lloyd iteration never reads another mesh's sites -- so N
GPUs run N independent engines with no data-path collective.  This module
holds the host-side pieces: a deterministic size-balanced partition of a mesh
list over ranks, and the max-over-ranks reduction of device times used when
reporting whole-job throughput.
"""
from __future__ import annotations

import heapq


def partition(sizes, world: int, rank: int):
    """Indices of the items rank `rank` owns out of `world`.

    Largest-first greedy onto the least loaded rank (ties by rank), so every
    rank computes the same assignment without communication and the loads
    differ by at most the largest item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    owner = [0] * len(sizes)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + sizes[i], r))
    return [i for i in range(len(sizes)) if owner[i] == rank]


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (e.g. device milliseconds) over the default
    process group; returns the value unchanged without one."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
