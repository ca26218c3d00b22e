"""Test-only driver for the reference library built from its own sources.

oracle/_ref/libffdas_ref.so is BrainEchoLab/ffdas's das path compiled for
sm_100a by `make -C oracle ref`.  Tests, the smoke check and bench.py's
reference leg call it through its C-ABI (include/ffdas.h of the reference) on
torch CUDA buffers, as a checker and as the speed bar.  Product code never
uses it.

Memory safety.  The reference kernel loads x[k] and x[k+1] for every unit
even when k is out of range (the weight is zeroed afterwards,
src/das/das_alg1_kernels.cuh:92-97), so a voxel outside the record reads
outside x.  Every call here therefore computes, on the host and in float64,
the full range of k the kernel can form for the given geometry, and places x
inside a larger buffer with that many guard elements on both sides.  Calls
whose range cannot be bounded this way are refused before the library is
entered.  Only ALG1 (reads the caller's buffer directly when x is contiguous
and already in the compute dtype) is driven with out-of-record voxels; ALG2
works on an internal permuted copy that cannot be guarded, so it is only
called when every k lies inside the record.
"""
from __future__ import annotations

import ctypes
import math
import os
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libffdas_ref.so"
MAX_GUARD = 1 << 26   # elements
_lib = None
_handles = {}

DT = {torch.float32: 0, torch.float16: 2, torch.float64: 16, torch.complex64: 4, torch.complex32: 6}


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(str(LIB_PATH), mode=ctypes.RTLD_LOCAL)
        vp = ctypes.c_void_p
        L.ffdas_create.argtypes = [ctypes.POINTER(vp)]
        L.ffdas_set_stream.argtypes = [vp, ctypes.c_size_t]
        L.ffdas_create_tensor_desc.argtypes = [ctypes.POINTER(vp), ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                               ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.ffdas_destroy_tensor_desc.argtypes = [vp]
        L.ffdas_das.argtypes = [vp, vp, vp, ctypes.c_float, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int]
        L.ffdas_das_sparse.argtypes = [vp, vp, vp, ctypes.c_float, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp,
                                       ctypes.c_int, ctypes.c_int]
        L.ffdas_truncate_rank.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_int64, vp, vp]
        L.ffdas_error_string.restype = ctypes.c_char_p
        _lib = L
    return _lib


def handle(device_index: int):
    h = _handles.get(device_index)
    if h is None:
        h = ctypes.c_void_p()
        rc = lib().ffdas_create(ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"reference ffdas_create failed: {rc}")
        _handles[device_index] = h
    return h


def _desc(dims, dtype_code):
    n = len(dims)
    d = ctypes.c_void_p()
    arr = (ctypes.c_int64 * n)(*dims)
    rc = lib().ffdas_create_tensor_desc(ctypes.byref(d), n, arr, None, dtype_code)
    if rc != 0:
        raise RuntimeError(f"reference desc failed {rc}")
    return d


def k_range(srcpos, dstpos, offsets) -> tuple[int, int]:
    """Smallest and largest floor(tau) the kernel can form (float64, with margin)."""
    sp = np.asarray(srcpos, np.float64).reshape(-1, 3)
    dp = np.asarray(dstpos, np.float64).reshape(-1, 3)
    # bounding boxes give a cheap, conservative distance range
    lo = np.maximum(0.0, np.maximum(sp.min(0)[None] - dp.max(0)[None], dp.min(0)[None] - sp.max(0)[None]))
    rmin = float(np.sqrt((lo ** 2).sum()))
    hi = np.maximum(np.abs(sp.max(0)[None] - dp.min(0)[None]), np.abs(dp.max(0)[None] - sp.min(0)[None]))
    rmax = float(np.sqrt((hi ** 2).sum()))
    o = np.asarray(offsets, np.float64)
    return int(math.floor(float(o.min()) + rmin)) - 2, int(math.floor(float(o.max()) + rmax)) + 2


def das(x: torch.Tensor, srcpos, dstpos, offsets, weights, *, sparse_indices=None, alg: int = 1,
        tile: int | None = None, srcdir=None, wavenum: float = 0.0, beta: complex = 0.0,
        out_init: torch.Tensor | None = None) -> torch.Tensor:
    """Reference das / das_sparse on a CUDA x (4-D, contiguous); returns (B, *spatial).

    x is copied into a guarded buffer first; the copy is outside any timing.
    srcdir (C, 4), wavenum (complex data) and beta are passed through as the
    reference's arguments; with beta != 0 the output starts from out_init.
    """
    assert x.is_cuda and x.ndim == 4
    dev = x.device
    B, C, S, N = x.shape
    kmin, kmax = k_range(srcpos.cpu().numpy(), dstpos.cpu().numpy(), offsets.cpu().numpy())
    guard = max(0, -kmin, kmax + 2 - N) + 64
    inside = kmin >= 0 and kmax <= N - 2
    if alg == 2 and not inside:
        raise ValueError("ALG2 reads an internal copy that cannot be guarded; every k must lie in the record")
    if guard > MAX_GUARD:
        raise ValueError(f"delay range needs {guard} guard elements; refusing to call the reference")
    if x.dtype == torch.complex32:   # complex half: a buffer of half pairs, viewed as complex32
        buf = torch.zeros(2 * (x.numel() + 2 * guard), dtype=torch.float16, device=dev).view(torch.complex32)
        xg = buf[guard:guard + x.numel()].view(x.shape)
        xg.view(torch.float16).copy_(x.contiguous().view(torch.float16))
    else:
        buf = torch.zeros(x.numel() + 2 * guard, dtype=x.dtype, device=dev)
        xg = buf[guard:guard + x.numel()].view(x.shape)
        xg.copy_(x)
    f32 = lambda t: t.to(device=dev, dtype=torch.float32).contiguous()  # noqa: E731
    srcpos, dstpos, offsets, weights = f32(srcpos), f32(dstpos), f32(offsets), f32(weights)
    sd = None if srcdir is None else f32(srcdir)
    spatial = tuple(dstpos.shape[:-1])
    out_dtype = torch.float64 if x.dtype == torch.float64 else (torch.complex64 if x.is_complex() else torch.float32)
    out = torch.zeros((B, *spatial), dtype=out_dtype, device=dev)
    if out_init is not None:
        out.copy_(out_init.reshape(out.shape))
    xd = _desc([B, C, S, N], DT[x.dtype])
    od = _desc([B, *spatial], DT[out_dtype])
    bc = complex(beta)
    beta = (ctypes.c_double * 2)(bc.real, bc.imag) if out_dtype == torch.float64 else \
        (ctypes.c_float * 2)(bc.real, bc.imag)
    h = handle(dev.index)
    L = lib()
    L.ffdas_set_stream(h, torch.cuda.current_stream(dev).cuda_stream)
    old = os.environ.get("FFDAS_ALG1_TILE_SIZE")
    if tile is not None:
        os.environ["FFDAS_ALG1_TILE_SIZE"] = str(tile)
    try:
        sdp = None if sd is None else sd.data_ptr()
        if sparse_indices is None:
            rc = L.ffdas_das(h, srcpos.data_ptr(), sdp, float(wavenum), xd, xg.data_ptr(), dstpos.data_ptr(),
                             offsets.data_ptr(), weights.data_ptr(), ctypes.cast(beta, ctypes.c_void_p), od,
                             out.data_ptr(), 0, alg)
        else:
            idx = sparse_indices.to(device=dev, dtype=torch.int32).contiguous()
            rc = L.ffdas_das_sparse(h, srcpos.data_ptr(), sdp, float(wavenum), xd, xg.data_ptr(), dstpos.data_ptr(),
                                    offsets.data_ptr(), weights.data_ptr(), int(idx.shape[0]), idx.data_ptr(),
                                    ctypes.cast(beta, ctypes.c_void_p), od, out.data_ptr(), 0, alg)
    finally:
        if tile is not None:
            if old is None:
                os.environ.pop("FFDAS_ALG1_TILE_SIZE", None)
            else:
                os.environ["FFDAS_ALG1_TILE_SIZE"] = old
        L.ffdas_destroy_tensor_desc(xd)
        L.ffdas_destroy_tensor_desc(od)
    if rc != 0:
        raise RuntimeError(f"reference ffdas_das failed: {L.ffdas_error_string(rc).decode()} ({rc})")
    torch.cuda.current_stream(dev).synchronize()
    del buf
    return out


class Prepared:
    """A reference call with guarded buffers allocated once, for timing loops."""

    def __init__(self, x: torch.Tensor, srcpos, dstpos, offsets, weights, *, sparse_indices=None, alg: int = 1,
                 tile: int | None = None):
        dev = x.device
        B, C, S, N = x.shape
        kmin, kmax = k_range(srcpos.cpu().numpy(), dstpos.cpu().numpy(), offsets.cpu().numpy())
        inside = kmin >= 0 and kmax <= N - 2
        if alg == 2 and not inside:
            raise ValueError("ALG2 needs every k inside the record")
        guard = max(0, -kmin, kmax + 2 - N) + 64
        if guard > MAX_GUARD:
            raise ValueError("delay range too large to guard")
        self.buf = torch.zeros(x.numel() + 2 * guard, dtype=x.dtype, device=dev)
        self.x = self.buf[guard:guard + x.numel()].view(x.shape)
        self.x.copy_(x)
        f32 = lambda t: t.to(device=dev, dtype=torch.float32).contiguous()  # noqa: E731
        self.srcpos, self.dstpos, self.offsets, self.weights = f32(srcpos), f32(dstpos), f32(offsets), f32(weights)
        self.idx = None if sparse_indices is None else sparse_indices.to(device=dev, dtype=torch.int32).contiguous()
        spatial = tuple(self.dstpos.shape[:-1])
        self.out = torch.zeros((B, *spatial), dtype=torch.float32, device=dev)
        self.xd = _desc([B, C, S, N], DT[x.dtype])
        self.od = _desc([B, *spatial], 0)
        self.beta = (ctypes.c_float * 2)()
        self.h = handle(dev.index)
        self.alg = alg
        self.tile = tile
        self.dev = dev

    def __call__(self):
        L = lib()
        L.ffdas_set_stream(self.h, torch.cuda.current_stream(self.dev).cuda_stream)
        if self.tile is not None:
            os.environ["FFDAS_ALG1_TILE_SIZE"] = str(self.tile)
        if self.idx is None:
            rc = L.ffdas_das(self.h, self.srcpos.data_ptr(), None, 0.0, self.xd, self.x.data_ptr(),
                             self.dstpos.data_ptr(), self.offsets.data_ptr(), self.weights.data_ptr(),
                             ctypes.cast(self.beta, ctypes.c_void_p), self.od, self.out.data_ptr(), 0, self.alg)
        else:
            rc = L.ffdas_das_sparse(self.h, self.srcpos.data_ptr(), None, 0.0, self.xd, self.x.data_ptr(),
                                    self.dstpos.data_ptr(), self.offsets.data_ptr(), self.weights.data_ptr(),
                                    int(self.idx.shape[0]), self.idx.data_ptr(), ctypes.cast(self.beta, ctypes.c_void_p),
                                    self.od, self.out.data_ptr(), 0, self.alg)
        if rc != 0:
            raise RuntimeError(f"reference call failed: {L.ffdas_error_string(rc).decode()}")
        return self.out

    def close(self):
        L = lib()
        L.ffdas_destroy_tensor_desc(self.xd)
        L.ffdas_destroy_tensor_desc(self.od)
        if self.tile is not None:
            os.environ.pop("FFDAS_ALG1_TILE_SIZE", None)


DT_RANK = {torch.float32: 0, torch.float64: 16, torch.complex64: 4, torch.complex128: 17}


class PreparedRank:
    """The reference's rank filter (src/truncate_rank/truncate_rank.cu:6-42) on a
    contiguous 2-D CUDA tensor, descriptors made once, for parity and timing.
    It reads x within its bounds, so no guard is needed; the window is checked
    here the way the reference's Python wrapper checks it."""

    def __init__(self, x: torch.Tensor, start: int, stop: int | None = None):
        if x.ndim != 2 or not x.is_contiguous() or x.dtype not in DT_RANK:
            raise ValueError("need a contiguous 2-D float32/float64/complex64/complex128 tensor")
        m, n = x.shape
        stop = min(m, n) if stop is None else stop
        if not (0 <= start < stop <= min(m, n)):
            raise ValueError("need 0 <= start < stop <= min(m, n)")
        self.x, self.start, self.stop = x, int(start), int(stop)
        self.out = torch.empty_like(x)
        self.xd = _desc([m, n], DT_RANK[x.dtype])
        self.od = _desc([m, n], DT_RANK[x.dtype])
        self.h = handle(x.device.index)
        self.dev = x.device

    def __call__(self):
        L = lib()
        L.ffdas_set_stream(self.h, torch.cuda.current_stream(self.dev).cuda_stream)
        rc = L.ffdas_truncate_rank(self.h, self.xd, self.x.data_ptr(), self.start, self.stop, self.od,
                                   self.out.data_ptr())
        if rc != 0:
            raise RuntimeError(f"reference truncate_rank failed: {L.ffdas_error_string(rc).decode()}")
        return self.out

    def close(self):
        L = lib()
        L.ffdas_destroy_tensor_desc(self.xd)
        L.ffdas_destroy_tensor_desc(self.od)


def truncate_rank(x: torch.Tensor, start: int, stop: int | None = None) -> torch.Tensor:
    call = PreparedRank(x.contiguous(), start, stop)
    try:
        return call().clone()
    finally:
        call.close()
