"""CPU check of the TMA-staged kernel's window arithmetic (no GPU).

Mirrors, in float32 numpy, how das_staged_kernel bounds the sample window of a
(voxel tile, channel, event) -- tile bounding box, min/max delay of the event
over the tile, floor(...) -/+ 2, x aligned down to 16 bytes -- and checks, on
the benchmark geometries, that every tap of every voxel of a tile falls inside
its staged window whenever the window is not flagged as overflow, and that the
TMA x coordinate is 16-byte aligned.
"""
import numpy as np
import pytest
import torch

from ffdas_b200 import workloads as W


def tiles_of(shape, T0=16, T1=16):
    D = [int(d) for d in shape if d != 1]
    D0 = D[-1]
    D1 = D[-2] if len(D) >= 2 else 1
    D2 = int(np.prod(D[:-2])) if len(D) > 2 else 1
    for t2 in range(D2):
        for t1 in range(0, D1, T1):
            for t0 in range(0, D0, T0):
                i1 = np.arange(t1, min(t1 + T1, D1))
                i0 = np.arange(t0, min(t0 + T0, D0))
                yield ((t2 * D1 + i1[:, None]) * D0 + i0[None, :]).ravel()


def check(wl, WB, pair_bytes=8, max_tiles=64, seed=0):
    dst = wl["dstpos"].reshape(-1, 3).numpy().astype(np.float32)
    src = wl["srcpos"].numpy().astype(np.float32)
    offs = wl["offsets"].reshape(wl["offsets"].shape[0], -1).numpy().astype(np.float32)
    N = wl["x"].shape[-1]
    npad = (max(N, 2) + 3) // 4 * 4
    align = 16 // pair_bytes
    tl = list(tiles_of(wl["dstpos"].shape[:-1]))
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(tl), min(max_tiles, len(tl)), replace=False)
    n_win = n_ovf = 0
    for ti in pick:
        vox = tl[ti]
        p = dst[vox]
        lo, hi = p.min(0), p.max(0)
        d = p[:, None, :] - src[None, :, :]
        rsq = np.maximum((d * d).sum(-1, dtype=np.float32), np.float32(1e-7))
        r = (rsq * (np.float32(1) / np.sqrt(rsq))).astype(np.float32)           # (v, c)
        dmin = np.maximum(np.maximum(lo[None] - src, src - hi[None]), 0).astype(np.float32)
        emax = np.maximum(np.abs(src - lo[None]), np.abs(src - hi[None])).astype(np.float32)
        rmin = np.sqrt((dmin * dmin).sum(-1, dtype=np.float32))
        rmax = np.sqrt((emax * emax).sum(-1, dtype=np.float32))
        for e in range(offs.shape[0]):
            o = offs[e, vox]
            wlo = np.floor(o.min() + rmin) - 2
            whi = np.floor(o.max() + rmax) + 2
            tau = (o[:, None] + r).astype(np.float32)                              # (v, c)
            k = np.floor(tau).astype(np.int64)
            for c in range(src.shape[0]):
                if not (whi[c] >= 0 and wlo[c] < npad):
                    # zero window: every tap must be out of the record
                    assert ((k[:, c] < 0) | (k[:, c] >= N - 1)).all()
                    continue
                k0 = int(max(wlo[c], -WB)) & ~(align - 1)
                k1 = int(min(whi[c], npad + WB))
                n_win += 1
                assert k0 % align == 0
                if k1 - k0 + 1 > WB:
                    n_ovf += 1
                    continue
                assert (k[:, c] >= k0).all() and (k[:, c] <= k1).all(), (e, c)
    return n_win, n_ovf


@pytest.mark.parametrize("WB", [32, 64])
def test_windows_cover_taps_diverging3d(WB):
    wl = W.diverging3d(scale=0.25)
    n, ovf = check(wl, WB)
    assert n > 0 and ovf / n < 0.5


def test_windows_cover_taps_plane2d():
    check(W.plane2d(scale=0.5), 64)


def test_windows_cover_taps_ensemble_fp16_pairs():
    wl = W.ensemble(scale=0.2, frames=2, dtype=torch.float32)
    check(wl, 32, pair_bytes=4)


def test_full_size_3d_volume_rarely_overflows():
    """At full size (16x16 tiles of the 128^3 volume) a 32-pair window holds
    nearly every (tile, channel, event) window."""
    wl = W.diverging3d(scale=1.0, n_side=8)   # 64 channels keep the check fast
    n, ovf = check(wl, 32, max_tiles=12)
    assert n > 0 and ovf / n < 0.05, (n, ovf)
