"""ffdas_das_static: the forward for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc at all -- a real-time or embedded host
that forbids allocation after start-up, or code that runs on a fixed memory
budget without an ffdas handle (whose creation allocates a workspace pool).
ffdas_das_static takes the caller's stream, inputs and output and keeps its
interpolation-pair workspace in a fixed array inside the library.  This test
calls it through the C-ABI and checks it against ffdas_das and against the
FP64 oracle on two calls in a row with different problem sizes (the second
call must not see the first call's leftovers), at the FP32 tolerance the
forward tests use (2e-5 relative L2; both library paths compute the same taps,
so their match is much closer), and that
a problem larger than the array is refused with FFDAS_ERROR_DIMS_TOO_LARGE.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone in a fresh process too.
"""
import ctypes

import pytest
import torch

import ffdas_b200
from ffdas_b200 import _lib, workloads as W
from ffdas_b200._lib import DataType, Error
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _static_call(wl, x):
    L = _lib.load()
    fn = L.ffdas_das_static
    vp = ctypes.c_void_p
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_size_t, vp, vp, ctypes.c_float, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int,
                   ctypes.c_int]
    out = torch.full((x.shape[0], *wl["dstpos"].shape[:-1]), float("nan"), device=DEV)
    x_desc = _lib.TensorDesc(list(x.shape), list(x.stride()), DataType.R_32F)
    o_desc = _lib.TensorDesc(list(out.shape), None, DataType.R_32F)
    beta = ctypes.c_float(0.0)
    rc = fn(torch.cuda.current_stream().cuda_stream, wl["srcpos"].data_ptr(), None, 0.0, x_desc.desc,
            x.data_ptr(), wl["dstpos"].data_ptr(), wl["offsets"].data_ptr(), wl["weights"].data_ptr(),
            ctypes.cast(ctypes.byref(beta), ctypes.c_void_p), o_desc.desc, out.data_ptr(), 0, 0)
    return rc, out


def test_static_workspace_matches_das_on_consecutive_calls():
    first = W.plane2d(device=DEV, scale=0.5)                 # 64 channels, 1 event, 1024 samples
    second = W.autofocus(device=DEV, scale=0.25, batch=2)    # 128 channels, 8 events, batch 2
    for wl in (first, second):
        x = wl["x"].float().contiguous()
        rc, got = _static_call(wl, x)
        assert rc == 0, _lib.error_string(rc)
        torch.cuda.synchronize()
        ref = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
        assert torch.isfinite(got).all()
        assert oracle.rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < 2e-5
        # and directly against the FP64 oracle, at the same bar
        exact = oracle.das_f64(x.cpu().numpy(), wl["srcpos"].cpu().numpy(), wl["dstpos"].cpu().numpy(),
                               wl["offsets"].cpu().numpy(), wl["weights"].cpu().numpy())
        assert oracle.rel_l2(got.cpu().numpy(), exact) < 2e-5


def test_static_workspace_refuses_oversized_problems():
    wl = W.diverging3d(device=DEV, scale=0.25)   # 64 ch x 4 events x 1024 samples x 8 B = 2 MiB: fits
    rc, _ = _static_call(wl, wl["x"].float().contiguous())
    assert rc == 0
    big = torch.zeros((1, 256, 16, 1024), device=DEV)       # 32 MiB of pairs: too large
    rc, _ = _static_call(dict(wl, x=big, srcpos=torch.zeros((256, 3), device=DEV)), big)
    assert rc == Error.DIMS_TOO_LARGE
