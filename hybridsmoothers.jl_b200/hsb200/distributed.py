"""Multi-GPU plumbing for the smoother path: one process per GPU.

The apply has no dependency between partitions and the served systems are
independent, so N GPUs run N replicas (or N disjoint shards of a request
stream) with no collective on the data path.  The only collectives are the
timing reduction (max over ranks, as the measurement rules require) and
result gathering on rank 0.
"""
from __future__ import annotations

import os


def rank_world():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def shard(items, rank, world):
    """Round-robin shard of a request list: rank r takes items r, r+world, ..."""
    return [it for i, it in enumerate(items) if i % world == rank]


def max_over_ranks(value, device=None):
    """Max of a float across the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
