"""C-ABI boundary: exported symbols, host-side behaviour and error codes.

CPU tests load libffdas_b200.so and exercise everything that needs no GPU;
the gpu-marked tests check that ffdas_das / ffdas_das_sparse return the
reference's error codes for the reference's invalid inputs
(src/das/das.cu:25-82, das_impl.cuh:34-54, das_utils.h:32-69,
das_alg1.cu:172-178, 267).
"""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest
import torch

from ffdas_b200 import _lib
from ffdas_b200._lib import Error, DataType

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "ffdas.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"FFDAS_API\s+[\w\s\*]+?\b(ffdas_\w+)\s*\(", text)))


def test_header_declares_the_das_path():
    names = declared_functions()
    for n in ("ffdas_das", "ffdas_das_sparse", "ffdas_create", "ffdas_destroy", "ffdas_set_stream",
              "ffdas_get_stream", "ffdas_create_tensor_desc", "ffdas_destroy_tensor_desc", "ffdas_error_string",
              "ffdas_type_size", "ffdas_event_create", "ffdas_event_elapsed_time", "ffdas_das_backward",
              "ffdas_truncate_rank"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH), mode=ctypes.RTLD_LOCAL)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_enum_values_match_reference():
    # include/ffdas.h:19-95 of the reference
    assert int(DataType.R_32F) == 0 and int(DataType.C_32F) == 4 and int(DataType.R_16F) == 2
    assert int(DataType.C_16F) == 6 and int(DataType.R_64F) == 16 and int(DataType.C_64F) == 17
    assert int(Error.INVALID_DIMS) == 2 and int(Error.DEVICE_MISMATCH) == 23 and int(Error.UNKNOWN) == 101
    text = HEADER.read_text()
    for name, val in [("FFDAS_ALG4", 4), ("FFDAS_COMPUTE_64F", 3), ("FFDAS_ERROR_CUDA_RUNTIME", 31),
                      ("FFDAS_R_16BF", 18), ("FFDAS_ERROR_OUT_OF_BOUNDS_INDEX", 63)]:
        assert re.search(rf"\b{name}\s*=\s*{val}\b", text), name


def test_error_strings_and_type_sizes():
    L = _lib.load()
    assert _lib.error_string(0) == "Success"
    assert _lib.error_string(2) == "Invalid dimensions"
    assert _lib.error_string(999) == "Unrecognized error code"
    sizes = {DataType.R_16F: 2, DataType.C_16F: 4, DataType.R_32F: 4, DataType.C_32F: 8, DataType.R_64F: 8,
             DataType.C_64F: 16, DataType.R_16I: 2, DataType.C_16I: 4, DataType.R_32I: 4, DataType.C_32I: 8,
             DataType.R_16BF: 2}
    for t, s in sizes.items():
        assert L.ffdas_type_size(int(t)) == s
    assert L.ffdas_type_size(99) == 0


def test_tensor_descriptor_validation():
    L = _lib.load()
    d = ctypes.c_void_p()
    dims = (ctypes.c_int64 * 2)(3, 4)
    assert L.ffdas_create_tensor_desc(None, 2, dims, None, 0) == Error.INVALID_ARGUMENT
    assert L.ffdas_create_tensor_desc(ctypes.byref(d), 0, dims, None, 0) == Error.INVALID_ARGUMENT
    assert L.ffdas_create_tensor_desc(ctypes.byref(d), 2, None, None, 0) == Error.INVALID_ARGUMENT
    assert L.ffdas_create_tensor_desc(ctypes.byref(d), 2, dims, None, 99) == Error.UNSUPPORTED_TYPE
    big = (ctypes.c_int64 * 17)(*([1] * 17))
    assert L.ffdas_create_tensor_desc(ctypes.byref(d), 17, big, None, 0) == Error.DIMS_TOO_LARGE
    assert L.ffdas_create_tensor_desc(ctypes.byref(d), 2, dims, None, 0) == 0
    assert L.ffdas_destroy_tensor_desc(d) == 0
    assert L.ffdas_destroy_tensor_desc(None) == 0


def test_null_handle_is_rejected_before_any_device_work():
    L = _lib.load()
    assert L.ffdas_das(None, None, None, 0.0, None, None, None, None, None, None, None, None, 0, 0) == \
        Error.INVALID_HANDLE
    assert L.ffdas_das_sparse(None, None, None, 0.0, None, None, None, None, None, 1, None, None, None, None,
                              0, 0) == Error.INVALID_HANDLE
    assert L.ffdas_das_backward(None, None, None, 0.0, None, None, None, None, None, 0, None, None, None, None,
                                None, None, None, None) == Error.INVALID_HANDLE
    assert L.ffdas_set_stream(None, 0) == Error.INVALID_HANDLE
    assert L.ffdas_get_stream(None, None) == Error.INVALID_HANDLE
    assert L.ffdas_destroy(None) == Error.INVALID_HANDLE
    assert L.ffdas_das_set_config(None, None) == Error.INVALID_HANDLE
    assert L.ffdas_sparse_select(None, None, None, 4, 16, 2, None, None, None) == Error.INVALID_HANDLE
    assert L.ffdas_truncate_rank(None, None, None, 0, 1, None, None) == Error.INVALID_HANDLE
    assert L.ffdas_contiguous_copy(None, None, None, None, None) == Error.INVALID_HANDLE
    assert L.ffdas_event_record(None, 1) == Error.INVALID_HANDLE
    assert L.ffdas_event_synchronize(0) == Error.INVALID_ARGUMENT
    assert L.ffdas_event_elapsed_time(0, 0, None) == Error.NULL_POINTER
    assert L.ffdas_event_destroy(0) == 0
    assert L.ffdas_device_count(None) == Error.NULL_POINTER


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_create_without_gpu_reports_an_error():
    L = _lib.load()
    h = ctypes.c_void_p()
    rc = L.ffdas_create(ctypes.byref(h))
    assert rc != 0 and not h.value
    assert L.ffdas_create(None) == Error.NULL_POINTER


# --------------------------------------------------------------------- GPU ---

def _call(handle, x_dims, x_dtype, out_dims, out_dtype, *, x_strides=None, compute=0, alg=0, sparse=None,
          ptrs=True):
    L = _lib.load()
    dev = "cuda:0"
    nx = int(np.prod(x_dims)) if len(x_dims) else 1
    x = torch.zeros(max(nx, 1) * 4, dtype=torch.float32, device=dev)
    out = torch.zeros(max(int(np.prod(out_dims)), 1) * 4, dtype=torch.float32, device=dev)
    buf = torch.zeros(1 << 16, dtype=torch.float32, device=dev)
    xd = _lib.TensorDesc(x_dims, x_strides, x_dtype)
    od = _lib.TensorDesc(out_dims, None, out_dtype)
    beta = (ctypes.c_double * 2)()
    p = buf.data_ptr() if ptrs else None
    if sparse is None:
        return L.ffdas_das(handle.h, p, None, 0.0, xd.desc, x.data_ptr() if ptrs else None, p, p, p,
                           ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr() if ptrs else None,
                           compute, alg)
    return L.ffdas_das_sparse(handle.h, p, None, 0.0, xd.desc, x.data_ptr(), p, p, p, sparse, p,
                              ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr(), compute, alg)


@pytest.mark.gpu
def test_error_codes_match_reference():
    import ffdas_b200
    h = ffdas_b200.get_library_handle("cuda:0")
    R32, R16, C32, R64 = DataType.R_32F, DataType.R_16F, DataType.C_32F, DataType.R_64F
    ok = ([1, 2, 2, 16], R32, [1, 4], R32)
    assert _call(h, *ok) == 0
    # dtype combination (das.cu:40-82)
    assert _call(h, [1, 2, 2, 16], R32, [1, 4], C32) == Error.UNSUPPORTED_TYPE
    assert _call(h, [1, 2, 2, 16], DataType.R_32I, [1, 4], R32) == Error.UNSUPPORTED_TYPE
    # x ndim (das_utils.h:39), batch mismatch (:52)
    assert _call(h, [2, 2, 16], R32, [4], R32) == 0
    assert _call(h, [2, 16], R32, [4], R32) == Error.INVALID_DIMS
    assert _call(h, [1, 1, 2, 2, 16], R32, [1, 4], R32) == Error.INVALID_DIMS
    assert _call(h, [2, 2, 2, 16], R32, [3, 4], R32) == Error.INVALID_DIMS
    # sample stride must be 1 (das_utils.h:66)
    assert _call(h, [1, 2, 2, 16], R32, [1, 4], R32, x_strides=[64, 32, 16, 2]) == Error.INVALID_ARGUMENT
    # int32 index guard (das_impl.cuh:34); size-1 dims do not count
    assert _call(h, [1, 2, 2, 16], R32, [1, 4], R32, x_strides=[1 << 31, 32, 16, 1]) == 0
    assert _call(h, [2, 2, 2, 16], R32, [2, 4], R32, x_strides=[1 << 31, 32, 16, 1]) == Error.INVALID_DIMS
    # algorithms: ALG3 is not implemented; fp64 only with ALG1/DEFAULT (das_impl.cuh:37-54)
    assert _call(h, *ok, alg=3) == Error.INVALID_ARGUMENT
    assert _call(h, *ok, alg=2) == 0
    assert _call(h, [1, 2, 2, 16], R64, [1, 4], R64, alg=2) == Error.UNSUPPORTED_TYPE
    # half input with a half compute request is rejected (das_alg1.cu:172-178)
    assert _call(h, [1, 2, 2, 16], R16, [1, 4], R32, compute=1) == Error.UNSUPPORTED_TYPE
    assert _call(h, [1, 2, 2, 16], R16, [1, 4], R32) == 0
    # sparse: count must be positive (das_alg1.cu:267), only ALG1/DEFAULT (das_sparse_impl.cuh:38-45)
    assert _call(h, *ok, sparse=0) == Error.INVALID_ARGUMENT
    assert _call(h, *ok, sparse=2) == 0
    assert _call(h, *ok, sparse=2, alg=2) == Error.INVALID_ARGUMENT
    # null data pointers are reported, never dereferenced
    assert _call(h, *ok, ptrs=False) == Error.NULL_POINTER
    # null descriptors
    L = _lib.load()
    assert L.ffdas_das(h.h, None, None, 0.0, None, None, None, None, None, None, None, None, 0, 0) == \
        Error.NULL_POINTER


@pytest.mark.gpu
def test_allocation_failure_is_reported_and_recoverable(rng):
    import ffdas_b200
    L = _lib.load()
    x = torch.randn((1, 3, 2, 64), device="cuda:0")
    src = torch.zeros((3, 3), device="cuda:0")
    dst = torch.rand((5, 3), device="cuda:0") + torch.tensor([0, 0, 10.0], device="cuda:0")
    offs = torch.rand((2, 5), device="cuda:0") * 10
    w = torch.ones((2, 5), device="cuda:0")
    from ffdas_b200.tune import schedule
    # the gather schedule stages pair rows in a workspace (the direct kernel
    # that small problems take by default allocates nothing)
    with schedule(dict(variant=1), "cuda:0"):
        good = ffdas_b200.das(x, src, dst, offs, w)
        L.ffdas_debug_fail_alloc_after(1)
        with pytest.raises(RuntimeError, match="Insufficient device memory"):
            ffdas_b200.das(x, src, dst, offs, w)
        again = ffdas_b200.das(x, src, dst, offs, w)
    assert torch.equal(good, again)


@pytest.mark.gpu
def test_device_mismatch_detected():
    import ffdas_b200
    h = ffdas_b200.get_library_handle("cuda:0")
    assert h.get_stream() is not None
    n = _lib.device_count()
    if n < 2:
        pytest.skip("one GPU")
    _lib.device_set(1)
    try:
        assert _call(h, [1, 2, 2, 16], DataType.R_32F, [1, 4], DataType.R_32F) == Error.DEVICE_MISMATCH
    finally:
        _lib.device_set(0)


@pytest.mark.gpu
def test_contiguous_copy_casts():
    import ffdas_b200
    h = ffdas_b200.get_library_handle("cuda:0")
    L = _lib.load()
    x = torch.randn((4, 6, 5), device="cuda:0").transpose(0, 2)   # non-contiguous (5, 6, 4)
    for odt, tdt, tol in [(DataType.R_32F, torch.float32, 0), (DataType.R_16F, torch.float16, 1e-3),
                          (DataType.R_16BF, torch.bfloat16, 1e-2), (DataType.R_64F, torch.float64, 0)]:
        out = torch.empty(x.shape, dtype=tdt, device="cuda:0")
        xd = _lib.TensorDesc(list(x.shape), list(x.stride()), DataType.R_32F)
        od = _lib.TensorDesc(list(out.shape), None, odt)
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        assert L.ffdas_contiguous_copy(h.h, xd.desc, x.data_ptr(), od.desc, out.data_ptr()) == 0
        torch.testing.assert_close(out.double(), x.double(), rtol=tol, atol=tol)
    bad = _lib.TensorDesc([5, 6], None, DataType.R_32F)
    xd = _lib.TensorDesc(list(x.shape), list(x.stride()), DataType.R_32F)
    assert L.ffdas_contiguous_copy(h.h, xd.desc, x.data_ptr(), bad.desc, x.data_ptr()) == Error.INVALID_DIMS
