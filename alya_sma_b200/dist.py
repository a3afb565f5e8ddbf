"""Multi-GPU host logic: one process per GPU (torchrun environment), the
batched ensemble sharded by specimens across ranks (no data-path
collective: specimens are independent), timings reduced as the max over
ranks.  Works with any torch.distributed backend (NCCL on GPUs, gloo for
the CPU tests)."""
from __future__ import annotations

import os


def env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def shard_specimens(sizes, rank, world):
    """Specimen ids of `rank`: longest-processing-time assignment by element
    count (largest first onto the least loaded rank, ties to the lowest rank),
    deterministic, a disjoint cover of range(len(sizes))."""
    order = sorted(range(len(sizes)), key=lambda s: (-int(sizes[s]), s))
    load = [0] * world
    owner = [0] * len(sizes)
    for s in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[s] = r
        load[r] += int(sizes[s])
    return [s for s in range(len(sizes)) if owner[s] == rank]


def max_over_ranks(value, device="cpu"):
    """Maximum of a float over all ranks (the slowest rank sets the time)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device="cpu"):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
