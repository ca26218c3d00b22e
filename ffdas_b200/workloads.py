"""Seeded synthetic delay-and-sum workloads with the shapes of the benchmark configs.

Every workload is a dict of torch tensors (x, srcpos, dstpos, offsets,
weights[, sparse_indices]) plus metadata.  Channel data is a sum of point
scatterers, each a Gaussian-enveloped cosine at 0.25 cycles/sample
(sigma = 3 samples) centred on its round-trip delay, plus N(0, noise) noise.
Positions are in sampling wavelengths, delays in samples (the reference's
units, docs/conventions.md).

  plane2d      128-ch linear array, 1 plane wave at 0 deg, B=1, N=2048, 256(z) x 128(x)
  diverging3d  32x32 matrix array, 16 diverging waves (virtual sources at z=-50 on a
               4x4 grid spanning +-12), B=1, N=4096, 128^3 voxels; separable Hann
               weights over the source grid: w = h(i) h(j), h(i) = sin^2(pi (i + 1/2) / 4)
  ensemble     200 frames x 128 ch x 11 plane waves (-10..10 deg) x 1536 samples,
               slow drift (0.01 samples/frame) plus 5% movers (0.3 samples/frame),
               400(z) x 256(x) voxels
  sparse_focus 64 focused transmits (foci on z = 800), each voxel using a seeded
               contiguous subset of 1-32 transmits (padded to 32 with weight 0)
  autofocus    128-ch linear array, 8 plane waves (-7..7 deg), B=4, N=2048, 256 x 256,
               data synthesised at sound-speed scale alpha = 1.03

`scale` < 1 shrinks channel count, event count, samples and grid together for
fast tests (same geometry family, seeded the same way).
"""
from __future__ import annotations

import math

import numpy as np
import torch

PULSE_F = 0.25     # cycles / sample
PULSE_SIGMA = 3.0  # samples


def _rf(tau: torch.Tensor, amp: torch.Tensor, n_samples: int, noise: float, gen: torch.Generator,
        dtype=torch.float32) -> torch.Tensor:
    """Sum of pulses: tau (..., P) round-trip delays -> (..., N) channel data."""
    dev = tau.device
    lead = tau.shape[:-1]
    P = tau.shape[-1]
    rows = int(np.prod(lead)) if len(lead) else 1
    half = int(math.ceil(4 * PULSE_SIGMA))
    j = torch.arange(-half, half + 1, device=dev, dtype=torch.float32)
    t = tau.reshape(rows, P, 1).float()
    n = torch.floor(t) + j                       # (rows, P, W)
    d = n - t
    val = torch.exp(-d * d / (2 * PULSE_SIGMA ** 2)) * torch.cos(2 * math.pi * PULSE_F * d)
    val = val * amp.reshape(1, P, 1).to(dev)
    ok = (n >= 0) & (n < n_samples)
    row = torch.arange(rows, device=dev).reshape(rows, 1, 1).expand_as(n)
    flat = (row * n_samples + n.clamp(0, n_samples - 1).long())[ok]
    out = torch.zeros(rows * n_samples, device=dev, dtype=torch.float32)
    out.index_add_(0, flat, val[ok])
    if noise > 0:
        out += noise * torch.randn(out.shape, generator=gen, device="cpu").to(dev)
    return out.reshape(*lead, n_samples).to(dtype)


def _linear_array(C: int, pitch: float = 1.0) -> torch.Tensor:
    xs = (torch.arange(C, dtype=torch.float32) - (C - 1) / 2) * pitch
    return torch.stack([xs, torch.zeros(C), torch.zeros(C)], -1)


def _grid2d(nz: int, nx: int, z0: float, z1: float, xhalf: float) -> torch.Tensor:
    z = torch.linspace(z0, z1, nz)
    x = torch.linspace(-xhalf, xhalf, nx)
    zz, xx = torch.meshgrid(z, x, indexing="ij")
    return torch.stack([xx, torch.zeros_like(xx), zz], -1)  # (nz, nx, 3)


def _n(v: int, scale: float, lo: int = 1) -> int:
    return max(lo, int(round(v * scale)))


def plane2d(device="cpu", scale: float = 1.0, seed: int = 0) -> dict:
    gen = torch.Generator().manual_seed(seed)
    C, N = _n(128, scale, 4), _n(2048, scale, 64)
    nz, nx = _n(256, scale, 2), _n(128, scale, 2)
    srcpos = _linear_array(C)
    P = 20
    px = (torch.rand(P, generator=gen) * 2 - 1) * 60 * scale
    pz = 200 * scale + torch.rand(P, generator=gen) * 1700 * scale
    pts = torch.stack([px, torch.zeros(P), pz], -1)
    rx = torch.cdist(srcpos, pts)                               # (C, P)
    tau = pz[None, None, :] + rx[:, None, :]                    # (C, 1, P)
    x = _rf(tau, torch.ones(P), N, 0.01, gen)[None]             # (1, C, 1, N)
    grid = _grid2d(nz, nx, 150 * scale, 1950 * scale, 64 * scale)  # (nz, nx, 3)
    dstpos = grid[:, None]                                       # (nz, 1, nx, 3)
    offsets = dstpos[..., 2][None].clone()                       # (1, nz, 1, nx)
    weights = torch.ones_like(offsets)
    d = dict(x=x, srcpos=srcpos, dstpos=dstpos, offsets=offsets, weights=weights)
    return _to(d, device, name="plane2d", scale=scale)


def diverging3d(device="cpu", scale: float = 1.0, seed: int = 1, n_side: int | None = None) -> dict:
    gen = torch.Generator().manual_seed(seed)
    side = n_side or _n(32, scale, 2)
    C = side * side
    N = _n(4096, scale, 64)
    nv = _n(128, scale, 2)
    e = torch.arange(side, dtype=torch.float32) - (side - 1) / 2
    ey, ex = torch.meshgrid(e, e, indexing="ij")
    srcpos = torch.stack([ex.reshape(-1), ey.reshape(-1), torch.zeros(C)], -1)
    g = torch.tensor([-12.0, -4.0, 4.0, 12.0])
    sy, sx = torch.meshgrid(g, g, indexing="ij")
    src = torch.stack([sx.reshape(-1), sy.reshape(-1), torch.full((16,), -50.0)], -1)  # (16, 3)
    S = 16 if scale >= 1 else max(2, min(16, _n(16, scale)))
    src = src[:S]
    h = torch.sin(math.pi * (torch.arange(4, dtype=torch.float32) + 0.5) / 4) ** 2
    hw = (h[:, None] * h[None, :]).reshape(-1)[:S]               # separable Hann over the 4x4 grid
    xy_half, z0, z1 = 40 * min(1.0, scale * 2), 100 * scale, 3900 * scale
    P = _n(200, scale, 4)
    pts = torch.stack([(torch.rand(P, generator=gen) * 2 - 1) * xy_half,
                       (torch.rand(P, generator=gen) * 2 - 1) * xy_half,
                       z0 + 100 * scale + torch.rand(P, generator=gen) * (z1 - z0 - 200 * scale)], -1)
    tx = torch.cdist(src, pts) - 50.0                            # (S, P)
    rx = torch.cdist(srcpos, pts)                                # (C, P)
    tau = tx[None] + rx[:, None]                                 # (C, S, P)
    x = _rf(tau.to(device), torch.ones(P), N, 0.01, gen)[None]   # (1, C, S, N)
    z = torch.linspace(z0, z1, nv)
    xy = torch.linspace(-xy_half, xy_half, nv)
    zz, yy, xx = torch.meshgrid(z, xy, xy, indexing="ij")
    dstpos = torch.stack([xx, yy, zz], -1)                       # (nz, ny, nx, 3)
    offsets = torch.cdist(src, dstpos.reshape(-1, 3)).reshape(S, nv, nv, nv) - 50.0
    weights = hw[:, None, None, None].expand(S, nv, nv, nv).contiguous()
    d = dict(x=x, srcpos=srcpos, dstpos=dstpos, offsets=offsets, weights=weights)
    return _to(d, device, name="diverging3d", scale=scale)


def normalize_channels(x: torch.Tensor) -> torch.Tensor:
    """Per-channel scale so each channel's peak |x| is 1 (precision-variant input)."""
    peak = x.abs().amax(dim=(-2, -1), keepdim=True).clamp_min(1e-30)
    return x / peak


def _plane_wave_delay(dstpos: torch.Tensor, theta: torch.Tensor) -> torch.Tensor:
    """x sin(theta) + z cos(theta) for every angle -> (S, *spatial)."""
    xx, zz = dstpos[..., 0], dstpos[..., 2]
    sh = (-1,) + (1,) * xx.ndim
    return xx[None] * torch.sin(theta).reshape(sh) + zz[None] * torch.cos(theta).reshape(sh)


def ensemble(device="cpu", scale: float = 1.0, seed: int = 3, frames: int | None = None,
             dtype=torch.float16) -> dict:
    gen = torch.Generator().manual_seed(seed)
    B = frames or _n(200, scale, 2)
    C, N = _n(128, scale, 4), _n(1536, scale, 64)
    S = 11 if scale >= 1 else max(2, _n(11, scale))
    nz, nx = _n(400, scale, 2), _n(256, scale, 2)
    theta = torch.deg2rad(torch.linspace(-10, 10, S))
    srcpos = _linear_array(C)
    P = _n(100, scale, 4)
    px = (torch.rand(P, generator=gen) * 2 - 1) * 60 * scale
    pz = 60 * scale + torch.rand(P, generator=gen) * 630 * scale
    movers = torch.rand(P, generator=gen) < 0.05
    rate = torch.where(movers, torch.tensor(0.3), torch.tensor(0.01)) / 2  # lambda/frame (round trip)
    frames_t = torch.arange(B, dtype=torch.float32)
    pzb = pz[None] + rate[None] * frames_t[:, None]              # (B, P)
    pts = torch.stack([px[None].expand(B, P), torch.zeros(B, P), pzb], -1)  # (B, P, 3)
    tx = (pts[..., 0][:, None] * torch.sin(theta)[None, :, None]
          + pts[..., 2][:, None] * torch.cos(theta)[None, :, None])     # (B, S, P)
    rx = torch.cdist(srcpos[None].expand(B, C, 3), pts)                 # (B, C, P)
    tau = tx[:, None] + rx[:, :, None]                                   # (B, C, S, P)
    x = _rf(tau.to(device), torch.ones(P), N, 0.01, gen, dtype=dtype)
    grid = _grid2d(nz, nx, 50 * scale, 700 * scale, 64 * scale)          # (nz, nx, 3)
    offsets = _plane_wave_delay(grid, theta)
    weights = torch.ones_like(offsets)
    d = dict(x=x, srcpos=srcpos, dstpos=grid, offsets=offsets, weights=weights)
    return _to(d, device, name="ensemble", scale=scale)


def sparse_focus(device="cpu", scale: float = 1.0, seed: int = 4, n_pad: int = 32) -> dict:
    gen = torch.Generator().manual_seed(seed)
    C, N = _n(128, scale, 4), _n(1536, scale, 64)
    T = 64 if scale >= 1 else max(4, _n(64, scale))
    n_pad = min(n_pad, T)
    nz, nx = _n(400, scale, 2), _n(256, scale, 2)
    srcpos = _linear_array(C)
    fx = torch.linspace(-60 * scale, 60 * scale, T)
    zf = 800.0 * scale
    foci = torch.stack([fx, torch.zeros(T), torch.full((T,), zf)], -1)
    P = _n(100, scale, 4)
    pts = torch.stack([(torch.rand(P, generator=gen) * 2 - 1) * 60 * scale, torch.zeros(P),
                       60 * scale + torch.rand(P, generator=gen) * 630 * scale], -1)

    def tx_delay(p):  # focused transmit: zf - / + distance to the focus
        dist = torch.cdist(foci, p)                              # (T, M)
        sign = torch.where(p[None, :, 2] < zf, -1.0, 1.0)
        return zf + sign * dist

    tau = tx_delay(pts)[None] + torch.cdist(srcpos, pts)[:, None]   # (C, T, P)
    x = _rf(tau.to(device), torch.ones(P), N, 0.01, gen)[None]      # (1, C, T, N)
    grid = _grid2d(nz, nx, 50 * scale, 700 * scale, 64 * scale)
    V = nz * nx
    full = tx_delay(grid.reshape(-1, 3))                            # (T, V)
    length = torch.randint(1, n_pad + 1, (V,), generator=gen)
    start = (torch.rand(V, generator=gen) * (T - length + 1).float()).long()
    i = torch.arange(n_pad)[:, None]
    valid = i < length[None]
    idx = torch.where(valid, start[None] + i, start[None]).int()    # repeated index on padding
    offsets = torch.gather(full, 0, idx.long())
    weights = valid.float()
    d = dict(x=x, srcpos=srcpos, dstpos=grid, offsets=offsets.reshape(n_pad, nz, nx),
             weights=weights.reshape(n_pad, nz, nx), sparse_indices=idx.reshape(n_pad, nz, nx))
    out = _to(d, device, name="sparse_focus", scale=scale)
    out["real_units"] = int(length.sum()) * C
    return out


def autofocus(device="cpu", scale: float = 1.0, seed: int = 5, alpha_true: float = 1.03,
              batch: int = 4) -> dict:
    """Sound-speed autofocus workload.

    The channel data is synthesised with every delay scaled by alpha_true
    (tau = alpha_true * (plane-wave delay + receive distance)); a beamformer
    with scale alpha uses positions alpha * p and delays alpha * base.  The
    scatterers lie in a shallow band (z 12..62) under the full 128-element
    aperture, where a 3% speed error visibly defocuses the image, so
    sharpness identifies alpha.  `scale` shrinks the grid and record only.
    """
    gen = torch.Generator().manual_seed(seed)
    B = batch
    C = 128
    N = _n(2048, scale, 512)
    S = 8
    nz, nx = _n(256, scale, 8), _n(256, scale, 8)
    theta = torch.deg2rad(torch.linspace(-7, 7, S))
    srcpos = _linear_array(C)
    P = 40
    frames = []
    for _ in range(B):
        pts = torch.stack([(torch.rand(P, generator=gen) * 2 - 1) * 40, torch.zeros(P),
                           12 + torch.rand(P, generator=gen) * 50], -1)
        tx = pts[:, 0][None] * torch.sin(theta)[:, None] + pts[:, 2][None] * torch.cos(theta)[:, None]
        tau = alpha_true * (tx[None] + torch.cdist(srcpos, pts)[:, None])
        frames.append(_rf(tau.to(device), torch.ones(P), N, 0.01, gen))
    x = torch.stack(frames)                                         # (B, C, S, N)
    grid = _grid2d(nz, nx, 6.0, 70.0, 48.0)
    base = _plane_wave_delay(grid, theta)
    d = dict(x=x, srcpos=srcpos, dstpos=grid, offsets=base, weights=torch.ones_like(base))
    out = _to(d, device, name="autofocus", scale=scale)
    out["alpha_true"] = alpha_true
    return out


def analytic_signal(x: torch.Tensor) -> torch.Tensor:
    """Analytic signal along the sample axis (FFT Hilbert transform), complex."""
    N = x.shape[-1]
    X = torch.fft.fft(x, dim=-1)
    h = torch.zeros(N, dtype=X.real.dtype, device=x.device)
    h[0] = 1
    h[1:(N + 1) // 2] = 2
    if N % 2 == 0:
        h[N // 2] = 1
    return torch.fft.ifft(X * h, dim=-1)


def _to(d: dict, device, **meta) -> dict:
    out = {k: v.to(device).contiguous() for k, v in d.items()}
    x = out["x"]
    B = x.shape[0] if x.ndim == 4 else 1
    C, S = x.shape[-3], x.shape[-2]
    V = int(np.prod(out["dstpos"].shape[:-1]))
    n_ev = out["offsets"].shape[0]
    out.update(meta)
    out["units"] = V * C * n_ev * B
    return out


def slow_time_ensemble(m: int, shape: tuple, dtype=torch.float32, device="cpu", seed: int = 51,
                       tissue: int = 5) -> torch.Tensor:
    """Seeded beamformed ensemble for the clutter filter (truncate_rank): m
    frames of `shape` voxels, `tissue` low-rank components each 4x weaker than
    the previous, plus weak full-rank 'blood' (1e-2).  Complex dtypes draw
    complex components (IQ images)."""
    g = torch.Generator().manual_seed(seed)
    n = 1
    for d in shape:
        n *= int(d)
    cplx = dtype.is_complex
    rdt = torch.float64

    def draw(*sz):
        a = torch.randn(*sz, generator=g, dtype=rdt)
        return torch.complex(a, torch.randn(*sz, generator=g, dtype=rdt)) if cplx else a

    u = torch.linalg.qr(draw(m, tissue))[0].to(device)
    v = (draw(n, tissue) / math.sqrt(n)).to(device)
    s = (10.0 * math.sqrt(n)) * 4.0 ** -torch.arange(tissue, dtype=rdt, device=device)
    x = (u * s) @ v.conj().T + 1e-2 * draw(m, n).to(device)
    return x.to(dtype).reshape(m, *shape).contiguous()


CONFIGS = {
    "plane2d": plane2d,
    "diverging3d": diverging3d,
    "ensemble": ensemble,
    "sparse_focus": sparse_focus,
    "autofocus": autofocus,
}
