"""Voxel sharding across ranks (one process per GPU).

Delay-and-sum voxels are independent, so a volume splits into slabs along its
outermost spatial dim with the channel data replicated on every rank; each
rank beamforms its slab with no collective on the data path.  `gather_slabs`
assembles the full image only when the caller wants one tensor
(torch.distributed.all_gather, any backend).  Frame ensembles shard the same
way along the batch dim (`shard_frames`).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def slab_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's share of n items, balanced to within one."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_voxels(dstpos, offsets, weights, rank: int, world: int, sparse_indices=None):
    """Rank's slab of the geometry along the outermost spatial dim (views, no copy)."""
    n = dstpos.shape[0]
    a, b = slab_bounds(n, rank, world)
    out = dict(dstpos=dstpos[a:b], offsets=offsets[:, a:b], weights=weights[:, a:b], slab=(a, b))
    if sparse_indices is not None:
        out["sparse_indices"] = sparse_indices[:, a:b]
    return out


def shard_frames(x, rank: int, world: int):
    """Rank's share of a (B, C, S, N) frame ensemble along the batch dim."""
    a, b = slab_bounds(x.shape[0], rank, world)
    return x[a:b], (a, b)


def gather_slabs(local: torch.Tensor, n_total: int, dim: int = 0, group=None) -> torch.Tensor:
    """All-gather uneven slabs along `dim` into the full image on every rank."""
    world = dist.get_world_size(group)
    sizes = [slab_bounds(n_total, r, world)[1] - slab_bounds(n_total, r, world)[0] for r in range(world)]
    biggest = max(sizes)
    shape = list(local.shape)
    shape[dim] = biggest
    padded = torch.zeros(shape, dtype=local.dtype, device=local.device)
    padded.narrow(dim, 0, local.shape[dim]).copy_(local)
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p.narrow(dim, 0, s) for p, s in zip(parts, sizes)], dim=dim)
