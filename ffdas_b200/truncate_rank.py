"""truncate_rank: keep the singular components start..stop-1 of an ensemble.

Mirrors the reference's Python function (bindings/python/ffdas/truncate_rank.py:28-91):
x (m, ...) is read as the matrix (m, prod(rest)), the output has x's shape,
and the arguments are checked the same way, with the same messages, before
the device is touched.  The work runs in ffdas_truncate_rank of
libffdas_b200.so (Gram matrix and projection kernels, cuSOLVER syevd).
"""
from __future__ import annotations

import math

import torch

from . import _lib
from ._lib import DataType
from .das import _from_torch_like, _to_torch
from .library import get_library_handle

_DTYPES = {
    torch.float32: DataType.R_32F,
    torch.float64: DataType.R_64F,
    torch.complex64: DataType.C_32F,
    torch.complex128: DataType.C_64F,
}


def truncate_rank(x, start: int, stop: int | None = None, *, out=None):
    """Rank truncation filter: reconstruct x from singular vectors start..stop-1.

    Args:
        x: CUDA array with at least 2 dimensions; float32, float64, complex64
            or complex128.  Read as the (m, n) matrix with m = x.shape[0].
        start: index of the first singular vector kept (0-based, descending
            singular values).
        stop: index past the last one kept; defaults to min(m, n).
        out: optional output of x's shape and dtype (may be x itself).

    Returns:
        The filtered array, of x's shape (``out`` when given).
    """
    if x.ndim < 2:
        raise ValueError(f"x must have at least 2 dimensions, got {x.ndim}")
    shp = tuple(x.shape)
    m = shp[0]
    n = math.prod(shp[1:])
    k = min(m, n)
    if start < 0 or start >= k:
        raise ValueError(f"start must be >= 0 and < min(m, n) ({m}, {n}), got {start}")
    if stop is None:
        stop = k
    elif stop <= start or stop > k:
        raise ValueError(f"stop must be > start ({start}) and <= min(m, n) ({m}, {n}), got {stop}")
    if out is not None and tuple(out.shape) != shp:
        raise ValueError("out must have the same dimensions as x")

    xt = _to_torch(x)
    if not xt.is_cuda:
        raise ValueError("x must be a CUDA array")
    if xt.dtype not in _DTYPES:
        raise TypeError(f"truncate_rank supports float32, float64, complex64 and complex128, got {xt.dtype}")
    dev = xt.device
    xc = xt.contiguous().view(m, n)
    ot = _to_torch(out) if out is not None else None
    if ot is not None:
        if ot.dtype != xt.dtype:
            raise TypeError(f"out has dtype {ot.dtype}, expected {xt.dtype}")
        if ot.device != dev:
            raise ValueError(f"out is on {ot.device}, expected {dev}")
    target = ot if ot is not None and ot.is_contiguous() else torch.empty(shp, dtype=xt.dtype, device=dev)
    dt = _DTYPES[xt.dtype]
    xd = _lib.TensorDesc((m, n), None, dt)
    od = _lib.TensorDesc((m, n), None, dt)
    handle = get_library_handle(dev)
    handle.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(_lib.load().ffdas_truncate_rank(handle.h, xd.desc, xc.data_ptr(), int(start), int(stop), od.desc,
                                               target.data_ptr()))
    if ot is not None:
        if target is not ot:
            ot.copy_(target)
        return out
    return _from_torch_like(target, x)
