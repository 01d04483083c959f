"""Independent scenes across GPUs: one process per GPU, scenes assigned to ranks
so that particle counts balance (longest-processing-time greedy). Scenes never
interact, so the data path has no collective; torch.distributed carries only the
barrier, the max-over-ranks timing and the final stats gather.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def assign_scenes(counts: Sequence[int], world: int) -> list:
    """Partition scene indices over `world` ranks, largest scene first onto the
    least-loaded rank. Returns one sorted index list per rank."""
    if world <= 0:
        raise ValueError("world must be positive")
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(counts)), key=lambda i: (-counts[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(counts[i]), r))
    return [sorted(x) for x in out]


def loads(counts: Sequence[int], parts: Sequence[Sequence[int]]) -> list:
    return [sum(int(counts[i]) for i in p) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float (timings are reported as the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_stats(stats: dict) -> list:
    """Every rank's stats dict, on every rank."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [stats]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, stats)
    return out
