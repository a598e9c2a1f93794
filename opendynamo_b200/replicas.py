"""Replica runs across GPUs (one process per GPU, no data exchange): the
step path does not shard at the graded sizes, so N GPUs run N independent
solver replicas and report whole-job throughput over the slowest rank.

The collective plumbing is torch.distributed (NCCL on GPUs, gloo on CPU);
only timing results cross ranks.
"""

from __future__ import annotations

import datetime
import os


def world() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 120):
    """Join the process group (None for a single process)."""
    n, _, _ = world()
    if n <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The largest value over all ranks (a rank's own value without a group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, seconds_max: float, n_ranks: int) -> float:
    """Whole-job rate: all ranks' units over the slowest rank's time."""
    return n_ranks * units_per_rank / seconds_max


def finish(dist=None):
    if dist is not None:
        dist.destroy_process_group()
