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


# ---------------------------------------------------------------------------
# 512-voxel kernel: pass skipping and the unclamped tap path (CPU mirror of
# pass_flags and staged_produce<FAST> in csrc/das_staged.cuh)

SANE = np.float32(1 << 20)


def check_fast(wl, WB, T0=32, T1=16, SC=8, pair_bytes=8, max_tiles=48, seed=0):
    """Per tile and pass: the skip rule may only skip passes whose every tap is
    outside the record; per window: a window the producer marks mappable must
    hold every tap of the tile (issued windows: [k0, k0 + WB - 1] of the
    pair row; zero windows: [lo, lo + WB - 1] of the zero slot).  Returns
    (passes, skipped, windows, mappable windows, stages, fast stages)."""
    dst = wl["dstpos"].reshape(-1, 3).numpy().astype(np.float32)
    src = wl["srcpos"].numpy().astype(np.float32)
    offs = wl["offsets"].reshape(wl["offsets"].shape[0], -1).numpy().astype(np.float32)
    S = offs.shape[0]
    N = wl["x"].shape[-1]
    npad = (max(N, 2) + 3) // 4 * 4
    align = 16 // pair_bytes
    cmin, cmax = src.min(0), src.max(0)
    tl = list(tiles_of(wl["dstpos"].shape[:-1], T0, T1))
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(tl), min(max_tiles, len(tl)), replace=False)
    stats = np.zeros(6, np.int64)
    CC = 32 // SC
    for ti in pick:
        vox = tl[ti]
        p = dst[vox]
        lo, hi = p.min(0), p.max(0)
        d = p[:, None, :] - src[None, :, :]
        rsq = np.maximum((d * d).sum(-1, dtype=np.float32), np.float32(1e-7))
        rinv = (np.float32(1) / np.sqrt(rsq)).astype(np.float32)
        r64 = rsq.astype(np.float64) * rinv.astype(np.float64)                    # exact product
        dmin_c = np.maximum(np.maximum(lo[None] - src, src - hi[None]), 0).astype(np.float32)
        emax_c = np.maximum(np.abs(src - lo[None]), np.abs(src - hi[None])).astype(np.float32)
        rmin = np.sqrt((dmin_c * dmin_c).sum(-1, dtype=np.float32))
        rmax = np.sqrt((emax_c * emax_c).sum(-1, dtype=np.float32))
        gap = np.maximum(np.maximum(cmin - hi, lo - cmax), 0).astype(np.float32)
        ext = np.maximum(np.abs(cmax - lo), np.abs(hi - cmin)).astype(np.float32)
        bmin, bmax = np.sqrt((gap * gap).sum(dtype=np.float32)), np.sqrt((ext * ext).sum(dtype=np.float32))
        for e0 in range(0, S, SC):
            evs = range(e0, min(S, e0 + SC))
            stats[0] += 1
            olo = [offs[e, vox].min() for e in evs]
            ohi = [offs[e, vox].max() for e in evs]
            skip = bmax <= SANE
            for a, b in zip(olo, ohi):
                marg = np.float32(4) + np.float32(1e-5) * (abs(a) + abs(b) + bmax)
                skip &= bool((a + bmin - marg >= N - 1) or (b + bmax + marg < 0))
            # fp32 tau as the kernel forms it: fma(rsq, rsqrt(rsq), offset)
            taus = {e: (offs[e, vox][:, None].astype(np.float64) + r64).astype(np.float32) for e in evs}
            ks = {e: np.floor(taus[e]).astype(np.int64) for e in evs}
            if skip:
                stats[1] += 1
                for e in evs:
                    assert ((ks[e] < 0) | (ks[e] >= N - 1)).all(), ("skipped pass has a tap in the record", e0)
                continue
            for c0 in range(0, src.shape[0], CC):
                stats[4] += 1
                all_map = True
                for cl in range(CC):
                    c = c0 + cl
                    for j in range(SC):
                        e = e0 + j
                        if c >= src.shape[0] or e >= S:
                            all_map = False
                            continue
                        wlo = np.floor(olo[j] + rmin[c]) - 2
                        whi = np.floor(ohi[j] + rmax[c]) + 2
                        sane = abs(wlo) <= SANE and abs(whi) <= SANE and rmax[c] <= SANE
                        k = ks[e][:, c]
                        stats[2] += 1
                        mappable = False
                        if whi >= 0 and wlo < npad:
                            k0 = int(max(wlo, -WB)) & ~(align - 1)
                            k1 = int(min(whi, npad + WB))
                            if k1 - k0 + 1 <= WB:
                                mappable = sane and k0 <= wlo and whi <= k0 + WB - 1
                                if mappable:
                                    assert (k >= k0).all() and (k <= k0 + WB - 1).all(), (e, c)
                        elif sane and whi - wlo + 1 <= WB:
                            mappable = True
                            kz = int(wlo)
                            assert (k >= kz).all() and (k <= kz + WB - 1).all(), (e, c)
                            assert ((k < 0) | (k >= N - 1)).all()
                        stats[3] += mappable
                        all_map &= mappable
                stats[5] += all_map
    return stats


def test_fast_path_and_skips_on_the_volume():
    """The headline volume's geometry (64 channels of the 32x32 array keep it
    fast): deep tiles skip whole passes, and most stages take the unclamped
    taps; every claim above is checked tap by tap."""
    wl = W.diverging3d(scale=1.0, n_side=8)
    st = check_fast(wl, 32, max_tiles=40)
    passes, skipped, wins, mapped, stages, fast = (int(v) for v in st)
    assert skipped > 0.3 * passes, st
    assert fast > 0.5 * stages, st


@pytest.mark.parametrize("WB", [32, 64])
def test_fast_path_windows_cover_taps_smaller_volume(WB):
    wl = W.diverging3d(scale=0.25)
    st = check_fast(wl, WB, T0=16, T1=32, SC=4, max_tiles=32, seed=1)
    assert st[0] > 0 and st[2] > 0


def test_fast_path_plane_wave_frame():
    wl = W.plane2d(scale=0.5)
    check_fast(wl, 64, T0=512, T1=1, SC=1, max_tiles=16)
