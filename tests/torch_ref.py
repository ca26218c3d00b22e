"""Pure-torch float64 delay-and-sum (CPU), differentiable: the autograd checker.

Same formula as the reference kernel (src/das/das_alg1_kernels.cuh:48-106):
tau = offsets[e,v] + sqrt(max(|dst[v]-src[c]|^2, 1e-7)), k = floor(tau),
t = tau - k, valid iff 0 <= k < N-1, out += w * (x[k] + t (x[k+1] - x[k])).
Gradients flow through t (not through the floor), exactly the derivative the
backward kernels implement.  Real data, or complex data with the phase
rotation out += w exp(i wavenum tau) L (src/das/das_alg1_kernels.cuh:79-86);
optional element directivity
(srcdir rows (nx, ny, nz, cos_min): a tap counts only where
(dst - src) . n / |dst - src| > cos_min, src/das/das_alg1_kernels.cuh:72-76),
a mask without gradient.  Small sizes only.
"""
from __future__ import annotations

import torch


def das_ref(x, srcpos, dstpos, offsets, weights, sparse_indices=None, srcdir=None, wavenum=0.0):
    """x ([B,] C, S, N); returns ([B,] *spatial) float64 (complex128 for complex x)."""
    have_batch = x.ndim == 4
    xb = x if have_batch else x[None]
    B, C, S, N = xb.shape
    spatial = dstpos.shape[:-1]
    V = dstpos[..., 0].numel()
    dp = dstpos.reshape(V, 3).double()
    sp = srcpos.reshape(C, 3).double()
    offs = offsets.reshape(-1, V).double()
    w = weights.reshape(-1, V).double()
    E = offs.shape[0]
    d = dp[:, None, :] - sp[None, :, :]                     # (V, C, 3)
    rsq = (d * d).sum(-1).clamp_min(1e-7)
    r = torch.sqrt(rsq)                                     # (V, C)
    tau = offs[:, :, None] + r[None]                        # (E, V, C)
    kf = torch.floor(tau.detach())
    t = tau - kf
    valid = (kf >= 0) & (kf < N - 1)
    if srcdir is not None:
        sd = srcdir.reshape(C, 4).double().detach()
        proj = (d.detach() * sd[None, :, :3]).sum(-1) / r.detach()     # (V, C)
        valid = valid & (proj > sd[None, :, 3])[None]
    k = kf.clamp(0, max(N - 2, 0)).long()
    if sparse_indices is None:
        s = torch.arange(E)[:, None, None].expand(E, V, C)
    else:
        s = sparse_indices.reshape(E, V).long()[:, :, None].expand(E, V, C)
        valid = valid & (s >= 0) & (s < S)
        s = s.clamp(0, S - 1)
    c = torch.arange(C)[None, None, :].expand(E, V, C)
    cplx = xb.is_complex()
    xd = xb.to(torch.complex128) if cplx else xb.double()
    phase = torch.exp(1j * float(wavenum) * tau) if cplx else None
    outs = []
    for b in range(B):
        x0 = xd[b][c, s, k]
        x1 = xd[b][c, s, (k + 1).clamp(max=N - 1)]
        L = x0 + t * (x1 - x0)
        if cplx:
            L = L * phase
        L = torch.where(valid, L, torch.zeros_like(L))
        outs.append((w[:, :, None] * L).sum(dim=(0, 2)))
    out = torch.stack(outs).reshape(B, *spatial)
    return out if have_batch else out[0]
