"""Python delay-and-sum API: `das` and `das_sparse`.

Signature, argument meaning and error behaviour mirror the reference's Python
API (bindings/python/ffdas/das.py:64-152 and :188-287): the same positional
order (x, srcpos, dstpos, offsets, weights[, sparse_indices]), the same
keywords (srcdir, wavenum, algorithm, use_fp16, channels_trailing, out), the
same ValueError shape checks before any GPU work (:107-123, :229-256), the same
float32/int32 casts with a DowncastWarning (bindings/python/ffdas/_core/
tensor.py:21-42), and RuntimeError(ffdas_error_string(code)) for a non-zero
library status (_ffdas.cpp:112-115).

Inputs may be torch CUDA tensors or any CUDA array exposing __dlpack__
(CuPy, JAX, ...): they are wrapped zero-copy with torch.from_dlpack.  The
result is a torch tensor, converted back through DLPack when x came from
another framework that offers from_dlpack.

Differences from the reference (documented, deliberate):
  * offsets/weights are indexed per event for 3-D x too (the reference reuses
    event 0's row when x has no batch dim);
  * the output of 16-bit real input is float32 and of complex32 input
    complex64 (the C-ABI's output dtypes);
  * int16 channel data (raw ADC samples) is accepted and interpolated in FP32
    (the reference's C-ABI has the int16 type code but rejects it for das);
  * `use_bf16=True` selects the new bf16 pair storage;
  * calls run on torch's current CUDA stream (the reference always uses the
    legacy default stream);
  * when autograd is on and an input requires grad, the call records a
    DASFunction node (ffdas_b200.autograd) with hand-written backward kernels.
"""
from __future__ import annotations

import ctypes
import sys
import warnings

import torch

from . import _lib
from ._lib import Algorithm, ComputeType, DataType
from .library import get_library_handle


class DowncastWarning(UserWarning):
    """Issued when an input is cast to the dtype the library requires."""


_FFDAS_DTYPE = {
    torch.float32: DataType.R_32F,
    torch.float16: DataType.R_16F,
    torch.bfloat16: DataType.R_16BF,
    torch.int16: DataType.R_16I,
    torch.float64: DataType.R_64F,
    torch.complex64: DataType.C_32F,
    torch.complex32: DataType.C_16F,
    torch.complex128: DataType.C_64F,
}
_OUT_DTYPE = {
    torch.float32: torch.float32,
    torch.float16: torch.float32,
    torch.bfloat16: torch.float32,
    torch.int16: torch.float32,
    torch.float64: torch.float64,
    torch.complex64: torch.complex64,
    torch.complex32: torch.complex64,
    torch.complex128: torch.complex128,
}


def _shape(a):
    return tuple(a.shape)


def _to_torch(a):
    if a is None or torch.is_tensor(a):
        return a
    if hasattr(a, "__dlpack__"):
        return torch.from_dlpack(a)
    return torch.as_tensor(a)


def _from_torch_like(out: torch.Tensor, like):
    """Return `out` in the array type of `like` when that is not torch."""
    if like is None or torch.is_tensor(like):
        return out
    mod = sys.modules.get(type(like).__module__.split(".")[0])
    conv = getattr(mod, "from_dlpack", None)
    if conv is None:
        return out
    try:
        return conv(out)
    except Exception:
        return out


def _astype(a, dtype: torch.dtype, device, name: str, stacklevel: int = 4):
    if a is None:
        return None
    t = _to_torch(a)
    if t.dtype != dtype:
        warnings.warn(f"input of type {t.dtype} will be downcast to {dtype}", DowncastWarning,
                      stacklevel=stacklevel)
        t = t.to(dtype)
    if t.device != device:
        raise ValueError(f"{name} is on {t.device}, expected {device}")
    return t.contiguous()


def _compute_type(x: torch.Tensor, use_fp16: bool, use_bf16: bool) -> ComputeType:
    # reference das.py:20-30, plus the bf16 pair storage
    if use_fp16:
        return ComputeType.FP16
    if use_bf16:
        return ComputeType.BF16
    if x.dtype in (torch.float64, torch.complex128):
        return ComputeType.FP64
    return ComputeType.FP32


def _x_desc(x: torch.Tensor, channels_trailing: bool) -> _lib.TensorDesc:
    dims = list(x.shape)
    strides = list(x.stride())
    if channels_trailing:
        # reference _ffdas.cpp:515-519: swap the channel and sequence dims
        c = 1 if x.ndim == 4 else 0
        dims[c], dims[c + 1] = dims[c + 1], dims[c]
        strides[c], strides[c + 1] = strides[c + 1], strides[c]
    return _lib.TensorDesc(dims, strides, _FFDAS_DTYPE[x.dtype])


def _beta_buffer(dtype: torch.dtype):
    n = 2 if dtype.is_complex else 1
    if dtype in (torch.float64, torch.complex128):
        return (ctypes.c_double * n)()
    return (ctypes.c_float * n)()


def _check_spatial(dstpos, offsets, weights, sparse_indices=None):
    if len(_shape(dstpos)) < 2 or _shape(dstpos)[-1] != 3:
        raise ValueError("dstpos must have dimensions (..., 3)")
    spatial = _shape(dstpos)[:-1]
    if _shape(offsets)[1:] != spatial:
        raise ValueError(f"offsets shape {_shape(offsets)} must match target layout {spatial}")
    if _shape(weights)[1:] != spatial:
        raise ValueError(f"weights shape {_shape(weights)} must match target layout {spatial}")
    if sparse_indices is not None:
        if _shape(sparse_indices)[1:] != spatial:
            raise ValueError(
                f"sparse_indices shape {_shape(sparse_indices)} must match target layout {spatial}")
        n = _shape(sparse_indices)[0]
        if _shape(offsets)[0] != n or _shape(weights)[0] != n:
            raise ValueError(f"offsets and weights leading dimension must match sparse count {n}")
    return spatial


def _needs_grad(*ts) -> bool:
    return torch.is_grad_enabled() and any(torch.is_tensor(t) and t.requires_grad for t in ts)


def _run(x, srcpos, dstpos, offsets, weights, sparse_indices, *, srcdir, wavenum, algorithm,
         use_fp16, use_bf16, channels_trailing, out, channel_scale=None, host_chunks=None):
    spatial = _check_spatial(dstpos, offsets, weights, sparse_indices)
    xt = _to_torch(x)
    if xt.ndim not in (3, 4):
        raise ValueError("x must have dimensions ([batch,] channels, sequence, samples)")
    if host_chunks is None:
        if not xt.is_cuda:
            raise ValueError("x must be a CUDA tensor")
        dev = xt.device
    else:
        if xt.is_cuda:
            raise ValueError("das_from_host takes x in host memory; use das for CUDA tensors")
        sp = _to_torch(srcpos)
        if not (torch.is_tensor(sp) and sp.is_cuda):
            raise ValueError("das_from_host needs srcpos, dstpos, offsets and weights on the GPU")
        dev = sp.device
        xt = xt.contiguous()
    if xt.dtype not in _FFDAS_DTYPE:
        raise TypeError(f"unsupported channel data dtype {xt.dtype}")
    srcpos_t = _astype(srcpos, torch.float32, dev, "srcpos")
    dstpos_t = _astype(dstpos, torch.float32, dev, "dstpos")
    offsets_t = _astype(offsets, torch.float32, dev, "offsets")
    weights_t = _astype(weights, torch.float32, dev, "weights")
    srcdir_t = _astype(srcdir, torch.float32, dev, "srcdir")
    idx_t = _astype(sparse_indices, torch.int32, dev, "sparse_indices") if sparse_indices is not None else None

    out_dims = tuple(spatial)
    if xt.ndim == 4:
        out_dims = (xt.shape[0], *out_dims)
    out_dtype = _OUT_DTYPE[xt.dtype]
    if out is None:
        out_t = torch.empty(out_dims, dtype=out_dtype, device=dev)
    else:
        out_t = _to_torch(out)
    beta = _beta_buffer(out_t.dtype)
    ctype = _compute_type(xt, use_fp16, use_bf16)

    handle = get_library_handle(dev)
    handle.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    x_desc = _x_desc(xt, channels_trailing)
    o_desc = _lib.TensorDesc(list(out_t.shape), list(out_t.stride()),
                             _FFDAS_DTYPE.get(out_t.dtype, DataType.R_32F))
    L = _lib.load()
    ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    scale_t = None
    if channel_scale is not None:
        scale_t = _astype(channel_scale, torch.float32, dev, "channel_scale")
        C = xt.shape[-2] if channels_trailing else xt.shape[-3]
        B = xt.shape[0] if xt.ndim == 4 else 1
        if scale_t.numel() not in (C, B * C):
            raise ValueError(f"channel_scale must hold {C} (per channel) or {B * C} (per item and channel) "
                             f"values, got shape {tuple(scale_t.shape)}")
        handle.set_channel_scale(scale_t.data_ptr(), scale_t.numel())
    try:
        if host_chunks is not None:
            code = L.ffdas_das_from_host(handle.h, ptr(srcpos_t), ptr(srcdir_t), float(wavenum), x_desc.desc,
                                         ptr(xt), ptr(dstpos_t), ptr(offsets_t), ptr(weights_t),
                                         ctypes.cast(beta, ctypes.c_void_p), o_desc.desc, ptr(out_t), int(ctype),
                                         int(algorithm), int(host_chunks))
        elif idx_t is None:
            code = L.ffdas_das(handle.h, ptr(srcpos_t), ptr(srcdir_t), float(wavenum), x_desc.desc, ptr(xt),
                               ptr(dstpos_t), ptr(offsets_t), ptr(weights_t), ctypes.cast(beta, ctypes.c_void_p),
                               o_desc.desc, ptr(out_t), int(ctype), int(algorithm))
        else:
            code = L.ffdas_das_sparse(handle.h, ptr(srcpos_t), ptr(srcdir_t), float(wavenum), x_desc.desc,
                                      ptr(xt), ptr(dstpos_t), ptr(offsets_t), ptr(weights_t), int(idx_t.shape[0]),
                                      ptr(idx_t), ctypes.cast(beta, ctypes.c_void_p), o_desc.desc, ptr(out_t),
                                      int(ctype), int(algorithm))
    finally:
        if scale_t is not None:
            handle.set_channel_scale(None, 0)
    _lib.check(code)
    if out is not None:
        return out
    return _from_torch_like(out_t, x)


def das_from_host(x, srcpos, dstpos, offsets, weights, *, srcdir=None, wavenum: float = 0.0,
                  algorithm: Algorithm = Algorithm.DEFAULT, use_fp16: bool = False, use_bf16: bool = False,
                  out=None, channel_scale=None, chunks: int = 0):
    """`das` on channel data in host memory (ffdas_das_from_host).

    x is a CPU tensor (or array), ([batch,] channels, sequence, samples), best
    in page-locked memory (`tensor.pin_memory()`) so that its upload overlaps
    the beamforming; every other tensor and the output are on the GPU.  The
    channels are uploaded in `chunks` runs (0: about channels / 128, at most
    8), each beamformed as soon as it has landed and added into the image, so
    only the first run's copy is not hidden.  The call returns once the work
    is queued on torch's current stream; x must stay unchanged until then.
    Same result as `das` up to the rounding of the sum over channels.  No
    autograd.
    """
    if _needs_grad(srcpos, dstpos, offsets, weights) or (torch.is_tensor(x) and x.requires_grad):
        raise NotImplementedError("das_from_host has no backward; use das on device data")
    if int(chunks) < 0:
        raise ValueError("chunks must be >= 0")
    return _run(x, srcpos, dstpos, offsets, weights, None, srcdir=srcdir, wavenum=wavenum, algorithm=algorithm,
                use_fp16=use_fp16, use_bf16=use_bf16, channels_trailing=False, out=out,
                channel_scale=channel_scale, host_chunks=int(chunks))


def das(x, srcpos, dstpos, offsets, weights, *, srcdir=None, wavenum: float = 0.0,
        algorithm: Algorithm = Algorithm.DEFAULT, use_fp16: bool = False, use_bf16: bool = False,
        channels_trailing: bool = False, out=None, channel_scale=None):
    """Delay-and-sum beamforming, compounding over the sequence dimension.

    For each target v:  out[b, v] = sum_s sum_c weights[s, v] *
    lerp(x[b, c, s, :], offsets[s, v] + |dstpos[v] - srcpos[c]|).
    Positions are in sampling wavelengths (c / fs), offsets in samples.

    Args:
        x: RF data, (channels, sequence, samples) or (batch, channels, sequence, samples);
            float32, float16, bfloat16, int16, float64, complex64, complex32 or complex128.
        srcpos: channel positions (channels, 3).
        dstpos: target positions (..., 3); the output has shape ([batch,] ...).
        offsets: per-target delays in samples (sequence, ...).
        weights: per-target apodization (sequence, ...).
        srcdir: optional (channels, 4): unit normal and cosine of the acceptance half-angle.
        wavenum: phase-rotation wavenumber for complex (IQ) data, e.g. -2*pi*fc/fs.
        algorithm: accepted for compatibility; the B200 planner picks the schedule.
        use_fp16: store channel data as fp16 pairs (fp32 interpolation and accumulation).
        use_bf16: store channel data as bf16 pairs (fp32 interpolation and accumulation).
        channels_trailing: x is ([batch,] sequence, channels, samples).
        out: optional preallocated output.
        channel_scale: optional per-channel scale, (channels,) or (batch, channels), applied
            to the channel data as it is stored (ffdas_set_channel_scale): e.g. 1 / peak to
            normalise each channel before fp16/bf16 storage, or ADC gains of int16 data.
            Not differentiable.
    """
    if _needs_grad(x, srcpos, dstpos, offsets, weights):
        if channel_scale is not None:
            raise NotImplementedError("channel_scale has no backward; apply the scale to x instead")
        from .autograd import das_autograd
        return das_autograd(x, srcpos, dstpos, offsets, weights, None, srcdir=srcdir, wavenum=wavenum,
                            use_fp16=use_fp16, use_bf16=use_bf16, channels_trailing=channels_trailing)
    return _run(x, srcpos, dstpos, offsets, weights, None, srcdir=srcdir, wavenum=wavenum, algorithm=algorithm,
                use_fp16=use_fp16, use_bf16=use_bf16, channels_trailing=channels_trailing, out=out,
                channel_scale=channel_scale)


def das_sparse(x, srcpos, dstpos, offsets, weights, sparse_indices, *, srcdir=None, wavenum: float = 0.0,
               algorithm: Algorithm = Algorithm.DEFAULT, use_fp16: bool = False, use_bf16: bool = False,
               channels_trailing: bool = False, out=None, channel_scale=None):
    """Sparse compounding: each target sums the n events named by sparse_indices (n, ...).

    Entries with weight exactly 0 are skipped, so per-target subsets of uneven
    length can be padded with weight 0.  Other arguments as in `das`.
    """
    if _needs_grad(x, srcpos, dstpos, offsets, weights):
        if channel_scale is not None:
            raise NotImplementedError("channel_scale has no backward; apply the scale to x instead")
        from .autograd import das_autograd
        return das_autograd(x, srcpos, dstpos, offsets, weights, sparse_indices, srcdir=srcdir,
                            wavenum=wavenum, use_fp16=use_fp16, use_bf16=use_bf16,
                            channels_trailing=channels_trailing)
    return _run(x, srcpos, dstpos, offsets, weights, sparse_indices, srcdir=srcdir, wavenum=wavenum,
                algorithm=algorithm, use_fp16=use_fp16, use_bf16=use_bf16, channels_trailing=channels_trailing,
                out=out, channel_scale=channel_scale)


def sparse_select(weights, k: int, offsets=None):
    """The inputs of `das_sparse`: per voxel the k events with the largest weight.

    Device version of the host step in the reference's sparse-compounding
    example (bindings/python/examples/sparse_compounding.py:141-144):
    ``sparse_indices = argpartition(weights, -k, axis=0)[-k:]`` and
    ``take_along_axis`` of the weights and delays at those indices.

    Args:
        weights: per-event apodization (n_events, ...), on a CUDA device.
        k: events kept per voxel, 1 <= k <= min(n_events, 32).
        offsets: optional per-event delays of the same shape, gathered too.

    Returns:
        (sparse_indices int32 (k, ...), sparse_weights (k, ...), sparse_offsets
        (k, ...) or None).  Entries come in descending weight (NaN above every
        number, ties to the lower event index); argpartition leaves that order
        unspecified, and das_sparse's sum depends on it only through rounding.
    """
    w_shape = _shape(weights)
    if len(w_shape) < 2:
        raise ValueError("weights must have dimensions (n_events, ...)")
    n = w_shape[0]
    if not isinstance(k, (int,)) or isinstance(k, bool):
        raise TypeError("k must be an int")
    if k < 1 or k > min(n, 32):
        raise ValueError(f"k must lie in [1, min(n_events, 32)] = [1, {min(n, 32)}], got {k}")
    if offsets is not None and _shape(offsets) != w_shape:
        raise ValueError(f"offsets shape {_shape(offsets)} must match weights shape {w_shape}")
    wt = _to_torch(weights)
    if not wt.is_cuda:
        raise ValueError("weights must be a CUDA tensor")
    dev = wt.device
    w_t = _astype(wt, torch.float32, dev, "weights")
    o_t = _astype(offsets, torch.float32, dev, "offsets") if offsets is not None else None
    spatial = w_shape[1:]
    V = 1
    for d in spatial:
        V *= int(d)
    idx = torch.empty((k, *spatial), dtype=torch.int32, device=dev)
    sw = torch.empty((k, *spatial), dtype=torch.float32, device=dev)
    so = torch.empty((k, *spatial), dtype=torch.float32, device=dev) if o_t is not None else None
    handle = get_library_handle(dev)
    handle.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    _lib.check(_lib.load().ffdas_sparse_select(handle.h, ptr(w_t), ptr(o_t), int(n), int(V), int(k), ptr(idx),
                                               ptr(sw), ptr(so)))
    return (_from_torch_like(idx, weights), _from_torch_like(sw, weights),
            None if so is None else _from_torch_like(so, weights))
