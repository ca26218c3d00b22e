"""torch.autograd.Function for delay-and-sum with hand-written backward kernels.

Forward calls ffdas_das / ffdas_das_sparse; backward calls ffdas_das_backward,
which recomputes each interpolation tap (no stored indices) and returns the
gradients with respect to channel data (two-tap adjoint scatter), weights,
delays (through the interpolant's slope) and voxel / channel positions.
Real channel data (float32, float16, bfloat16) without phase rotation, and
complex IQ data (complex64, complex32) with any wavenum; element directivity
(srcdir) masks taps as in the forward, and the mask has no gradient (it is
piecewise constant in the positions).  The gradient of x is returned in x's
dtype and layout.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import DataType
from .das import _FFDAS_DTYPE, _astype, _check_spatial, _compute_type, _run, _to_torch, _x_desc
from .library import get_library_handle


def _backward_supported(x: torch.Tensor, wavenum: float) -> bool:
    if x.is_complex():
        return x.dtype in (torch.complex64, torch.complex32)
    return wavenum == 0.0 and x.dtype in (torch.float32, torch.float16, torch.bfloat16, torch.int16)


class DASFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, srcpos, dstpos, offsets, weights, sparse_indices, opts: dict):
        ctx.opts = opts
        ctx.pairs = None
        xt = x.detach()
        handle = get_library_handle(xt.device)
        # The forward builds its interpolation-pair rows into a buffer kept for
        # the backward (ffdas_set_pair_buffer), which then skips building them
        # again; only where the backward can run.
        keep = _backward_supported(xt, opts["wavenum"])
        if keep:
            nbytes = _lib.pair_bytes(_x_desc(xt, opts["channels_trailing"]), _compute_type(xt, False, False))
            ctx.pairs = torch.empty(nbytes, dtype=torch.uint8, device=xt.device)
            handle.set_pair_buffer(ctx.pairs.data_ptr(), nbytes)
        try:
            out = _run(xt, srcpos.detach(), dstpos.detach(), offsets.detach(), weights.detach(),
                       sparse_indices, srcdir=opts["srcdir"], wavenum=opts["wavenum"], algorithm=0,
                       use_fp16=opts["use_fp16"], use_bf16=opts["use_bf16"],
                       channels_trailing=opts["channels_trailing"], out=None)
        finally:
            if keep:
                handle.set_pair_buffer(None, 0)
        ctx.save_for_backward(x, srcpos, dstpos, offsets, weights,
                              sparse_indices if sparse_indices is not None else torch.empty(0))
        ctx.has_sparse = sparse_indices is not None
        return out

    @staticmethod
    def backward(ctx, gout):
        x, srcpos, dstpos, offsets, weights, idx = ctx.saved_tensors
        opts = ctx.opts
        if not _backward_supported(x, opts["wavenum"]):
            raise NotImplementedError("das backward supports real data without phase rotation (wavenum 0) "
                                      "and complex64 / complex32 data")
        need = ctx.needs_input_grad
        dev = x.device
        cplx = x.is_complex()
        gout = gout.contiguous().to(torch.complex64 if cplx else torch.float32)
        xt = x.detach()
        lead = xt.shape if xt.ndim == 4 else (1, *xt.shape)
        if opts["channels_trailing"]:
            B, S, C, N = lead
        else:
            B, C, S, N = lead
        gx = torch.zeros((B, C, S, N), dtype=torch.complex64 if cplx else torch.float32, device=dev) if need[0] else None
        goff = torch.empty(offsets.shape, dtype=torch.float32, device=dev) if need[3] else None
        gw = torch.empty(weights.shape, dtype=torch.float32, device=dev) if need[4] else None
        gdst = torch.empty(dstpos.shape, dtype=torch.float32, device=dev) if need[2] else None
        gsrc = torch.empty(srcpos.shape, dtype=torch.float32, device=dev) if need[1] else None

        dims = list(xt.shape)
        strides = list(xt.stride())
        if opts["channels_trailing"]:
            c = 1 if xt.ndim == 4 else 0
            dims[c], dims[c + 1] = dims[c + 1], dims[c]
            strides[c], strides[c + 1] = strides[c + 1], strides[c]
        x_desc = _lib.TensorDesc(dims, strides, _FFDAS_DTYPE[xt.dtype])
        g_desc = _lib.TensorDesc(list(gout.shape), list(gout.stride()), DataType.C_32F if cplx else DataType.R_32F)
        f32 = lambda t: _astype(t.detach(), torch.float32, dev, "input")  # noqa: E731
        srcpos_t, dstpos_t, offsets_t, weights_t = f32(srcpos), f32(dstpos), f32(offsets), f32(weights)
        srcdir_t = f32(_to_torch(opts["srcdir"])) if opts["srcdir"] is not None else None
        idx_t = _astype(idx, torch.int32, dev, "sparse_indices") if ctx.has_sparse else None
        handle = get_library_handle(dev)
        handle.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        if ctx.pairs is not None:   # the forward's pair rows, read instead of rebuilt when they match
            handle.set_pair_buffer(ctx.pairs.data_ptr(), ctx.pairs.numel())
        try:
            _lib.check(_lib.load().ffdas_das_backward(
                handle.h, ptr(srcpos_t), ptr(srcdir_t), float(opts["wavenum"]), x_desc.desc, ptr(xt), ptr(dstpos_t),
                ptr(offsets_t),
                ptr(weights_t), int(idx_t.shape[0]) if idx_t is not None else 0, ptr(idx_t), g_desc.desc,
                ptr(gout), ptr(gx), ptr(goff), ptr(gw), ptr(gdst), ptr(gsrc)))
        finally:
            if ctx.pairs is not None:
                handle.set_pair_buffer(None, 0)
        ctx.pairs = None
        if gx is not None:
            if opts["channels_trailing"]:
                gx = gx.transpose(1, 2)
            if xt.ndim == 3:
                gx = gx[0]
            gx = gx.to(xt.dtype)
        cast = lambda g, ref: None if g is None else g.to(ref.dtype)  # noqa: E731
        return gx, cast(gsrc, srcpos), cast(gdst, dstpos), cast(goff, offsets), cast(gw, weights), None, None


def das_autograd(x, srcpos, dstpos, offsets, weights, sparse_indices=None, *, srcdir=None, wavenum=0.0,
                 use_fp16=False, use_bf16=False, channels_trailing=False):
    """Differentiable das / das_sparse (see ffdas_b200.das)."""
    _check_spatial(dstpos, offsets, weights, sparse_indices)
    tens = [_to_torch(t) for t in (x, srcpos, dstpos, offsets, weights)]
    idx = _to_torch(sparse_indices) if sparse_indices is not None else None
    opts = dict(srcdir=srcdir, wavenum=float(wavenum), use_fp16=use_fp16, use_bf16=use_bf16,
                channels_trailing=channels_trailing)
    return DASFunction.apply(*tens, idx, opts)
