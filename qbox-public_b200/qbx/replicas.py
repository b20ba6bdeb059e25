"""Independent replicas over several GPUs (one process per GPU).

The electronic step of one system does not shard in this library: several
GPUs run independent systems (the same cell on every GPU for the weak-scaling
bench, or a batch of small cells split across GPUs), with no collective on
the data path.  This module holds the bookkeeping around that: the rank
environment set by torchrun, the process group (NCCL between GPUs, gloo on
CPU), the partition of independent systems, and the max-over-ranks reduction
of a timing.
"""
from __future__ import annotations

import os
from datetime import timedelta
from typing import List, Tuple


def dist_env() -> Tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 600.0) -> None:
    """Join the process group of a multi-process run (no-op for one rank)."""
    import torch.distributed as dist
    _, world, _ = dist_env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def shard(n: int, rank: int, world: int) -> List[int]:
    """The indices of n independent systems this rank steps: contiguous
    blocks, sizes differing by at most one, every index on exactly one rank."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def max_over_ranks(x: float, device=None) -> float:
    """The largest value of x over the ranks (the job's time is its slowest
    rank's); x itself for one rank."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None) -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        if device is not None and str(device).startswith("cuda"):
            dist.barrier(device_ids=[int(str(device).split(":")[1])])
        else:
            dist.barrier()


def finalize() -> None:
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
