"""Multi-GPU plumbing for depth-map jobs: one process per GPU.

Reference views are independent units of work for the photometric pass, so a
scene's views are sharded across ranks with no data-path collective. The
geometric pass of a view reads its source views' photometric depth maps; when
a scene is split across ranks those maps are exchanged once, between the two
passes (``all_gather_maps``). Timing is the max over ranks.
"""
from __future__ import annotations

import numpy as np


def shard(num_items: int, world: int, rank: int) -> list:
    """Balanced contiguous split of range(num_items) for `rank` of `world`."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"bad rank {rank} of world {world}")
    base, extra = divmod(num_items, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value: float) -> float:
    """Max of `value` over all ranks (identity without a process group)."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(value)
    import torch
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_gather_maps(local: dict) -> dict:
    """Exchange per-view maps ({view index: array}) so every rank holds all of
    them (the step between the photometric and the geometric pass)."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, {int(k): np.asarray(v) for k, v in local.items()})
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise ValueError(f"view {k} produced on two ranks")
            merged[k] = v
    return merged
