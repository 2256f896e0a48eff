"""Multi-GPU layouts of the projector pair, one process per GPU.

Replicas (every workload that fits one GPU): each rank takes its own slices
or jobs and no data crosses ranks (``bench.py`` and
``serving.scheduler.shard``).

View-split back projection (one cone volume whose back projection should be
shared by several GPUs): rank r back projects views r, r + W, r + 2W, ... of
the scan into a full-volume partial sum; a reduce-scatter (sum) then leaves
each rank the z slab it owns, and an all-gather rebuilds the volume where the
next forward projection needs all of it.  The collectives run over NCCL on
GPUs (NVLink / NVSwitch; NCCL may reduce inside the switch) and over gloo on
CPU tensors.  The back projection itself is any callable, e.g. the Siddon
back projector applied to the geometry rows of the rank's views.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import torch
import torch.distributed as dist


def view_shares(nview: int, rank: int, world: int) -> List[int]:
    """The views rank ``rank`` of ``world`` back projects (round robin, so every
    rank sees the whole angular range)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(range(rank, nview, world))


def z_slabs(nz: int, world: int) -> List[Tuple[int, int]]:
    """Slice range [z0, z1) owned by each rank: equal slabs of ceil(nz / world)
    slices (the last ones may be short or empty)."""
    per = -(-nz // world)
    return [(min(nz, r * per), min(nz, (r + 1) * per)) for r in range(world)]


def _group_info(group):
    return dist.get_rank(group), dist.get_world_size(group)


def view_split_bp(bp_views: Callable[[Sequence[int]], torch.Tensor], nview: int, group=None
                  ) -> Tuple[torch.Tensor, Tuple[int, int]]:
    """Back projection of one volume split over the ranks of ``group`` by views.

    ``bp_views(views)`` returns this rank's partial back projection
    [nz, ny, nx] (float32) of the listed views.  Returns the rank's z slab of
    the sum over all views and its slice range."""
    rank, world = _group_info(group)
    partial = bp_views(view_shares(nview, rank, world))
    if partial.dim() != 3:
        raise ValueError("bp_views must return a [nz, ny, nx] volume")
    nz, ny, nx = partial.shape
    per = -(-nz // world)
    if per * world != nz:
        pad = torch.zeros((per * world - nz, ny, nx), dtype=partial.dtype, device=partial.device)
        partial = torch.cat([partial, pad])
    slab = torch.empty((per, ny, nx), dtype=partial.dtype, device=partial.device)
    dist.reduce_scatter_tensor(slab, partial.contiguous(), op=dist.ReduceOp.SUM, group=group)
    z0, z1 = z_slabs(nz, world)[rank]
    return slab[: z1 - z0], (z0, z1)


def gather_slabs(slab: torch.Tensor, nz: int, group=None) -> torch.Tensor:
    """The whole volume from every rank's z slab (as returned by
    ``view_split_bp``)."""
    rank, world = _group_info(group)
    per = -(-nz // world)
    ny, nx = slab.shape[1:]
    buf = torch.zeros((per, ny, nx), dtype=slab.dtype, device=slab.device)
    buf[: slab.shape[0]] = slab
    full = torch.empty((per * world, ny, nx), dtype=slab.dtype, device=slab.device)
    dist.all_gather_into_tensor(full, buf, group=group)
    return full[:nz]
