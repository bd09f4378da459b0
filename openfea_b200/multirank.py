"""Host-side logic of multi-GPU runs (one process per GPU).

The single-matrix solve does not shard; the batched reanalysis does: its
variants are independent, so each rank solves a subset with its own
persistent kernel and the ranks exchange nothing but the final statistics.
"""
from __future__ import annotations

import heapq


def partition_variants(costs, world):
    """Longest-first onto the least-loaded rank (ties: lower rank, then lower
    variant index).  Returns one ascending list of variant indices per rank;
    every rank computes the same partition from the same costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def max_over_ranks(x, dist=None, device=None):
    """The largest value of x over all ranks (timings are reported as the max)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    if device is None:
        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_by_variant(local, dist=None):
    """Merge per-rank {variant index: stats} dicts on every rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, dict(local))
    merged = {}
    for d in out:
        for k, v in d.items():
            if k in merged:
                raise RuntimeError(f"variant {k} solved on two ranks")
            merged[k] = v
    return merged
