"""Replica bookkeeping for multi-GPU runs.

Assembly of one mesh is not sharded across GPUs (the reference assembles on one
device and there is no inter-GPU exchange on the path): N ranks run independent
replicas, one process per GPU, and a step takes as long as the slowest rank.
The process group is used only for the barrier around the timed region and the
max-reduction of the per-rank step time.
"""
from __future__ import annotations

import datetime
import os


def init_from_env(backend: str = "nccl", timeout_s: int = 600):
    """(world, rank, local_rank, group or None) from the torchrun environment."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return 1, 0, 0, None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local, dist


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The maximum of `value` over all ranks (the value itself on one rank)."""
    if group is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    group.all_reduce(t, op=group.ReduceOp.MAX)
    return float(t.item())


def barrier(group=None) -> None:
    if group is not None:
        group.barrier()
