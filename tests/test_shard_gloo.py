"""Multi-rank path on CPU: world_size-2 gloo ranks each beamform their voxel slab
(the FP64 oracle stands in for the GPU kernel, which needs no collective) and
assemble the image with gather_slabs; the result must equal the single-rank
image exactly.  Also checks the slab arithmetic for uneven splits."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ffdas_b200.shard import gather_slabs, shard_frames, shard_voxels, slab_bounds


def test_slab_bounds_cover_exactly():
    for n in (1, 7, 128, 401):
        for world in (1, 2, 3, 8):
            spans = [slab_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    g = torch.Generator().manual_seed(3)
    B, C, S, N, nz, nx = 2, 5, 3, 96, 7, 6
    x = torch.randn((B, C, S, N), generator=g)
    src = torch.zeros((C, 3))
    src[:, 0] = torch.linspace(-3, 3, C)
    zz, xx = torch.meshgrid(torch.linspace(20, 40, nz), torch.linspace(-3, 3, nx), indexing="ij")
    dst = torch.stack([xx, torch.zeros_like(xx), zz], -1)
    offs = torch.rand((S, nz, nx), generator=g) * 30
    w = torch.rand((S, nz, nx), generator=g)
    return x, src, dst, offs, w


def _worker(rank, world, port, q):
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, src, dst, offs, w = _problem()
        sh = shard_voxels(dst, offs, w, rank, world)
        local = oracle.das_f64(x.numpy(), src.numpy(), sh["dstpos"].numpy(), sh["offsets"].numpy(),
                               sh["weights"].numpy())
        full = gather_slabs(torch.from_numpy(np.ascontiguousarray(local)), dst.shape[0], dim=1)
        xf, (a, b) = shard_frames(x, rank, world)
        framed = oracle.das_f64(xf.numpy(), src.numpy(), dst.numpy(), offs.numpy(), w.numpy())
        frames = gather_slabs(torch.from_numpy(np.ascontiguousarray(framed)), x.shape[0], dim=0)
        if rank == 0:
            q.put((full.numpy(), frames.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_assemble_the_single_rank_image():
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, frames = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    x, src, dst, offs, w = _problem()
    ref = oracle.das_f64(x.numpy(), src.numpy(), dst.numpy(), offs.numpy(), w.numpy())
    np.testing.assert_array_equal(full, ref)
    np.testing.assert_array_equal(frames, ref)
