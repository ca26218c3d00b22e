"""Test-only checkers: ctypes wrappers around oracle/_build/liboracle.so.

This module is test infrastructure.  Only tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py use it, and only as the checker; no product
code path imports it.

  das_f64(...)   FP64 restatement of the reference kernel das_alg1_kernel
                 (src/das/das_alg1_kernels.cuh:16-107), see das_oracle.c.
  das_f32(...)   the same formula as a plain FP32 OpenMP loop (CPU baseline).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
_lib = None


def build() -> Path:
    """Compile liboracle.so with the Makefile next to this file if missing or stale."""
    src = HERE / "das_oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "all"], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        p = ctypes.c_void_p
        L.oracle_das_f64.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                     p, ctypes.c_int, p, p, ctypes.c_float, p, p, p, ctypes.c_int, p,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_double, p]
        L.oracle_das_f64.restype = None
        L.oracle_das_f32.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                     p, p, p, p, p, p]
        L.oracle_das_f32.restype = None
        L.oracle_num_threads.restype = ctypes.c_int
        L.oracle_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def num_threads() -> int:
    return lib().oracle_num_threads()


def set_num_threads(n: int) -> None:
    lib().oracle_set_num_threads(int(n))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return None if a is None else np.ascontiguousarray(np.asarray(a), dtype=np.float32)


def das_f64(x, srcpos, dstpos, offsets, weights, *, srcdir=None, wavenum=0.0,
            sparse_indices=None, beta=0.0, out=None, channels_trailing=False, q1=False):
    """FP64 delay-and-sum of numpy inputs; returns float64 or complex128.

    Shapes follow the reference's Python das (bindings/python/ffdas/das.py:64):
    x ([B,] C, S, N), srcpos (C, 3), dstpos (..., 3), offsets/weights
    (n, ...), sparse_indices (n, ...) or None.  q1=True reproduces the
    reference's event-0 indexing for 3-D x.
    """
    x = np.asarray(x)
    have_batch = x.ndim == 4
    if not have_batch:
        x = x[None]
    if channels_trailing:
        x = np.swapaxes(x, 1, 2)
    B, C, S, N = x.shape
    cplx = np.iscomplexobj(x)
    xd = np.ascontiguousarray(x, dtype=np.complex128 if cplx else np.float64)
    if cplx:
        xd = np.ascontiguousarray(xd.view(np.float64).reshape(B, C, S, N, 2))
    dstpos = _f32(dstpos)
    spatial = dstpos.shape[:-1]
    V = int(np.prod(spatial)) if len(spatial) else 1
    offs = _f32(offsets).reshape(-1, V)
    wts = _f32(weights).reshape(-1, V)
    n_events = offs.shape[0] if sparse_indices is not None else S
    idx = None
    if sparse_indices is not None:
        idx = np.ascontiguousarray(np.asarray(sparse_indices), dtype=np.int32).reshape(-1, V)
    res = np.zeros((B, V, 2) if cplx else (B, V), dtype=np.float64)
    if out is not None:
        o = np.asarray(out)
        if not have_batch:
            o = o[None]
        o = o.reshape(B, V)
        res[...] = np.stack([o.real, o.imag], -1) if cplx else o.real
    bc = complex(beta)
    lib().oracle_das_f64(B, C, S, N, V, _ptr(xd), int(cplx), _ptr(_f32(srcpos)), _ptr(_f32(srcdir)),
                         float(wavenum), _ptr(dstpos), _ptr(offs), _ptr(wts), int(n_events), _ptr(idx),
                         int(bool(q1) and not have_batch), bc.real, bc.imag, _ptr(res))
    if cplx:
        res = res[..., 0] + 1j * res[..., 1]
    res = res.reshape((B, *spatial))
    return res if have_batch else res[0]


def das_f32(x, srcpos, dstpos, offsets, weights):
    """FP32 CPU loop (real, dense, beta = 0).  x is (B, C, S, N) float32."""
    x = np.ascontiguousarray(np.asarray(x), dtype=np.float32)
    have_batch = x.ndim == 4
    if not have_batch:
        x = x[None]
    B, C, S, N = x.shape
    dstpos = _f32(dstpos)
    spatial = dstpos.shape[:-1]
    V = int(np.prod(spatial))
    out = np.zeros((B, V), dtype=np.float32)
    lib().oracle_das_f32(B, C, S, N, V, _ptr(x), _ptr(_f32(srcpos)), _ptr(dstpos),
                         _ptr(_f32(offsets).reshape(-1, V)), _ptr(_f32(weights).reshape(-1, V)), _ptr(out))
    out = out.reshape((B, *spatial))
    return out if have_batch else out[0]


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def error_report(test, ref) -> dict:
    """rel-L2, peak abs error and peak error in dB below the reference's max."""
    test = np.asarray(test)
    ref = np.asarray(ref)
    err = np.abs(test.astype(np.complex128) - ref.astype(np.complex128))
    peak = float(err.max()) if err.size else 0.0
    ref_max = float(np.abs(ref).max()) if ref.size else 0.0
    db = float(20 * np.log10(peak / ref_max)) if peak > 0 and ref_max > 0 else float("-inf")
    return {"rel_l2": rel_l2(test, ref), "peak_abs": peak, "peak_db_below_max": db}
