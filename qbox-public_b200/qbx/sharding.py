"""Band pairs of one cell split over GPUs (one process per GPU).

The FFT work of an electronic step - update_density and the local part of
H*psi - is independent per band pair, as it is over the reference's state
axis (nstb of MPIdata::set, src/MPIdata.cpp:55-121).  Each rank's context
holds the whole cell and coefficients; qbx_set_band_shard gives it a
contiguous range of band pairs (qbx_shard_pairs), the library sums the
density over the ranks and gathers the H*psi bands from their owners with
NCCL, and every rank then runs the same products on the same data.

This module creates the NCCL group: rank 0 makes the id with
qbx_nccl_unique_id and the torch.distributed process group carries it to
the other ranks.
"""
from __future__ import annotations

from typing import List, Tuple

from . import capi


def pair_ranges(nst: int, world: int) -> List[Tuple[int, int]]:
    """[(first_pair, end_pair)] of every rank, from the library's own rule."""
    return [capi.shard_pairs(nst, r, world) for r in range(world)]


def band_ranges(nst: int, world: int) -> List[Tuple[int, int]]:
    """[(first_band, end_band)] of every rank (pair p = bands 2p, 2p+1)."""
    return [(2 * a, min(2 * b, nst)) for a, b in pair_ranges(nst, world)]


def shard_band_pairs(ctx, device=None) -> Tuple[int, int]:
    """Split ctx's band pairs over the ranks of the current process group
    (every rank calls this with its own context of the same cell).  Returns
    (rank, world)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return 0, 1
    rank, world = dist.get_rank(), dist.get_world_size()
    uid = capi.nccl_unique_id() if rank == 0 else bytes(capi.NCCL_ID_BYTES)
    t = torch.tensor(list(uid), dtype=torch.uint8)
    if device is not None and dist.get_backend() == "nccl":
        t = t.to(device)
    dist.broadcast(t, src=0)
    ctx.set_band_shard(rank, world, bytes(t.cpu().tolist()))
    return rank, world
