"""Replica plumbing for decoding one capture per GPU (one process per GPU).

The decode path has no data exchange between GPUs: captures (and fields
once their line locations are known) are independent, so N GPUs run N
replicas and the only collective is the max of the per-rank elapsed times
that a benchmark reports.  Rank layout comes from the environment torchrun
sets (RANK, WORLD_SIZE, LOCAL_RANK).
"""

import os


def dist_env():
    """(rank, world_size, local_rank) from the launcher's environment."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def capture_seed(base, rank):
    """Each replica decodes its own synthetic capture."""
    return int(base) + int(rank)


def max_over_ranks(value, world, device="cpu"):
    """The largest `value` over all ranks (every rank gets it); `value`
    itself when there is one rank.  Collective: every rank must call it."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
