"""Several GPUs of one node, one process per GPU (torchrun; RANK, WORLD_SIZE,
LOCAL_RANK from the environment).

One GSE-k system does not shard without an all-to-all FFT and a halo exchange
of the spread and gather, so a single system runs as independent replicas.  A
batch of independent systems is partitioned across the ranks: each rank
evaluates its own share, and nothing crosses GPUs on the data path.  The only
collectives are the barriers around timed regions and the reduction of each
rank's device time to the maximum over ranks, which every rank calls in the
same order.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def system_cost(n: int, grid: Sequence[int]) -> float:
    """Relative cost of one system in a batched evaluation: the spread and
    gather scale with the charges (about 2,900 stencil points each), the FFT
    solve with the grid points (a few operations each)."""
    return float(n) + 0.1 * float(grid[0]) * float(grid[1]) * float(grid[2])


def partition_systems(costs: Sequence[float], world: int) -> List[List[int]]:
    """Split systems 0..len(costs)-1 over `world` ranks: longest first onto the
    least-loaded rank (ties to the lower rank), each rank's list in ascending
    order.  Deterministic, so every rank computes the same partition without
    communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over the ranks of the default process group (the
    value itself without one).  Every rank must call it at the same point."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    """dist.barrier() when a process group with more than one rank exists."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
