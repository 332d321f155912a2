"""Replica plumbing for multi-GPU runs.

A reconstruction never spans GPUs (one fits in one B200's memory), so N GPUs
run N independent replicas: one process per GPU, launched by torchrun, with
torch.distributed used only to line the ranks up (barrier) and to take the
slowest rank's time.  Works with the NCCL backend on GPUs and gloo on CPU.
"""
from __future__ import annotations

import os


def world():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 600.0) -> bool:
    """Initialises the process group when more than one rank runs."""
    import datetime

    import torch.distributed as dist

    ws, _, _ = world()
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws > 1


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (every rank gets it)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(n_ranks: int, steps: int, max_seconds: float) -> float:
    """Whole-job units per second: every rank processed `steps` units."""
    return n_ranks * steps / max_seconds


def shutdown() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
