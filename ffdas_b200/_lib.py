"""ctypes binding of libffdas_b200.so (the C-ABI in include/ffdas.h).

Mirrors what the reference's nanobind module provides for the delay-and-sum
path (bindings/python/ffdas/_core/src/_ffdas.cpp): error checking that turns a
non-zero ffdas_error_t into RuntimeError(ffdas_error_string(code))
(:112-115), a Handle owning an ffdas_handle_t (:118), scoped tensor
descriptors, enums (:308-323) and the event/device helpers.  The library is
loaded from the package directory (or FFDAS_B200_LIB); there is no fallback:
if it is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes
import enum
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("FFDAS_B200_LIB", _PKG / "libffdas_b200.so"))

c_handle = ctypes.c_void_p
c_desc = ctypes.c_void_p
c_ptr = ctypes.c_void_p
c_err = ctypes.c_int


class DataType(enum.IntEnum):
    R_16F = 2
    C_16F = 6
    R_32F = 0
    C_32F = 4
    R_64F = 16
    C_64F = 17
    R_32I = 10
    C_32I = 11
    R_16I = 14
    C_16I = 15
    R_16BF = 18


class ComputeType(enum.IntEnum):
    DEFAULT = 0
    FP16 = 1
    FP32 = 2
    FP64 = 3
    BF16 = 4


class Algorithm(enum.IntEnum):
    DEFAULT = 0
    ALG1 = 1
    ALG2 = 2
    ALG3 = 3
    ALG4 = 4


class Error(enum.IntEnum):
    SUCCESS = 0
    INVALID_ARGUMENT = 1
    INVALID_DIMS = 2
    UNSUPPORTED_TYPE = 3
    NULL_POINTER = 4
    INVALID_HANDLE = 5
    NON_CONTIGUOUS = 6
    DIMS_TOO_LARGE = 7
    ALLOCATION_FAILED = 10
    DEVICE_MEMORY_INSUFFICIENT = 11
    HOST_MEMORY_INSUFFICIENT = 12
    INVALID_DEVICE = 13
    DEVICE_NOT_SUPPORTED = 20
    INSUFFICIENT_COMPUTE_CAPABILITY = 21
    DEVICE_NOT_AVAILABLE = 22
    DEVICE_MISMATCH = 23
    CUDA_DRIVER = 30
    CUDA_RUNTIME = 31
    CUDA_LAUNCH_FAILED = 32
    CUDA_SYNC_FAILED = 33
    CUDA_MEMCPY_FAILED = 34
    INVALID_STATE = 62
    INTERNAL = 100
    UNKNOWN = 101


class DasConfig(ctypes.Structure):
    """ffdas_das_config_t: schedule override (0 = planner default)."""
    _fields_ = [("variant", ctypes.c_int32), ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32),
                ("tile_z", ctypes.c_int32), ("batch_tile", ctypes.c_int32), ("event_chunk", ctypes.c_int32),
                ("min_blocks", ctypes.c_int32), ("window", ctypes.c_int32), ("copy_engine", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class KernelInfo(ctypes.Structure):
    """ffdas_kernel_info_t: what the last call launched."""
    _fields_ = [("variant", ctypes.c_int32), ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32),
                ("tile_z", ctypes.c_int32), ("batch_tile", ctypes.c_int32), ("event_chunk", ctypes.c_int32),
                ("storage", ctypes.c_int32), ("kernels", ctypes.c_int32), ("grid", ctypes.c_int64),
                ("copy_engine", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


# name -> (restype, argtypes)
SIGNATURES = {
    "ffdas_type_size": (ctypes.c_size_t, [ctypes.c_int]),
    "ffdas_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "ffdas_create_tensor_desc": (c_err, [ctypes.POINTER(c_desc), ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int64), ctypes.c_int]),
    "ffdas_destroy_tensor_desc": (c_err, [c_desc]),
    "ffdas_create": (c_err, [ctypes.POINTER(c_handle)]),
    "ffdas_destroy": (c_err, [c_handle]),
    "ffdas_set_stream": (c_err, [c_handle, ctypes.c_size_t]),
    "ffdas_get_stream": (c_err, [c_handle, ctypes.POINTER(ctypes.c_size_t)]),
    "ffdas_contiguous_copy": (c_err, [c_handle, c_desc, c_ptr, c_desc, c_ptr]),
    "ffdas_das": (c_err, [c_handle, c_ptr, c_ptr, ctypes.c_float, c_desc, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr,
                          c_desc, c_ptr, ctypes.c_int, ctypes.c_int]),
    "ffdas_das_sparse": (c_err, [c_handle, c_ptr, c_ptr, ctypes.c_float, c_desc, c_ptr, c_ptr, c_ptr, c_ptr,
                                 ctypes.c_int, c_ptr, c_ptr, c_desc, c_ptr, ctypes.c_int, ctypes.c_int]),
    "ffdas_das_backward": (c_err, [c_handle, c_ptr, c_ptr, ctypes.c_float, c_desc, c_ptr, c_ptr, c_ptr, c_ptr,
                                   ctypes.c_int, c_ptr, c_desc, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr]),
    "ffdas_sparse_select": (c_err, [c_handle, c_ptr, c_ptr, ctypes.c_int, ctypes.c_int64, ctypes.c_int, c_ptr,
                                    c_ptr, c_ptr]),
    "ffdas_truncate_rank": (c_err, [c_handle, c_desc, c_ptr, ctypes.c_int64, ctypes.c_int64, c_desc, c_ptr]),
    "ffdas_das_set_config": (c_err, [c_handle, ctypes.POINTER(DasConfig)]),
    "ffdas_das_get_config": (c_err, [c_handle, ctypes.POINTER(DasConfig)]),
    "ffdas_get_last_kernel_info": (c_err, [c_handle, ctypes.POINTER(KernelInfo)]),
    "ffdas_device_count": (c_err, [ctypes.POINTER(ctypes.c_int)]),
    "ffdas_device_get": (c_err, [ctypes.POINTER(ctypes.c_int)]),
    "ffdas_device_set": (c_err, [ctypes.c_int]),
    "ffdas_event_create": (c_err, [ctypes.POINTER(ctypes.c_size_t)]),
    "ffdas_event_destroy": (c_err, [ctypes.c_size_t]),
    "ffdas_event_record": (c_err, [c_handle, ctypes.c_size_t]),
    "ffdas_event_synchronize": (c_err, [ctypes.c_size_t]),
    "ffdas_event_elapsed_time": (c_err, [ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(ctypes.c_float)]),
    "ffdas_debug_fail_alloc_after": (None, [ctypes.c_int]),
    "ffdas_set_kernel_timing": (c_err, [c_handle, ctypes.c_int]),
    "ffdas_get_last_kernel_time": (c_err, [c_handle, ctypes.POINTER(ctypes.c_float)]),
    "ffdas_get_last_kernel_units": (c_err, [c_handle, ctypes.POINTER(ctypes.c_longlong)]),
    "ffdas_set_channel_scale": (c_err, [c_handle, c_ptr, ctypes.c_int64]),
    "ffdas_set_gram_engine": (c_err, [c_handle, ctypes.c_int32]),
    "ffdas_das_from_host": (c_err, [c_handle, c_ptr, c_ptr, ctypes.c_float, c_desc, c_ptr, c_ptr, c_ptr, c_ptr,
                                    c_ptr, c_desc, c_ptr, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "ffdas_set_pair_buffer": (c_err, [c_handle, c_ptr, ctypes.c_size_t]),
    "ffdas_das_pair_bytes": (c_err, [c_desc, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "ffdas_measure_fp32_peak": (c_err, [c_handle, ctypes.POINTER(ctypes.c_double)]),
    "ffdas_get_device_status": (c_err, [c_handle, ctypes.POINTER(ctypes.c_int)]),
    "ffdas_debug_staged_drop_stage": (None, [ctypes.c_int]),
}

_lib = None


def load(path: Path | str | None = None):
    """Load the library (once) and attach signatures.  Raises ImportError if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"libffdas_b200.so not found at {p}; build it with `python ffdas_b200/build.py` "
            "(nvcc for sm_100a is required; there is no CPU fallback)")
    lib = ctypes.CDLL(str(p), mode=ctypes.RTLD_LOCAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def error_string(code: int) -> str:
    return load().ffdas_error_string(int(code)).decode()


class FFDASError(RuntimeError):
    """RuntimeError carrying the ffdas_error_t code."""

    def __init__(self, code: int):
        self.code = int(code)
        super().__init__(error_string(self.code))


def check(code: int) -> None:
    if code != 0:
        raise FFDASError(code)


class TensorDesc:
    """Scoped ffdas_tensor_desc_t (dims and strides in elements)."""

    def __init__(self, dims, strides, dtype: int):
        n = len(dims)
        self._dims = (ctypes.c_int64 * n)(*[int(d) for d in dims])
        self._strides = (ctypes.c_int64 * n)(*[int(s) for s in strides]) if strides is not None else None
        self.desc = c_desc()
        check(load().ffdas_create_tensor_desc(ctypes.byref(self.desc), n, self._dims, self._strides, int(dtype)))

    def __del__(self):
        try:
            if self.desc:
                load().ffdas_destroy_tensor_desc(self.desc)
                self.desc = c_desc()
        except Exception:
            pass


class Handle:
    """Owns one ffdas_handle_t for the current device (reference _ffdas.cpp:118)."""

    def __init__(self):
        self.h = c_handle()
        check(load().ffdas_create(ctypes.byref(self.h)))

    def set_stream(self, stream: int) -> None:
        check(load().ffdas_set_stream(self.h, int(stream)))

    def get_stream(self) -> int:
        s = ctypes.c_size_t()
        check(load().ffdas_get_stream(self.h, ctypes.byref(s)))
        return int(s.value)

    def set_config(self, cfg: DasConfig | dict | None) -> None:
        if cfg is None:
            check(load().ffdas_das_set_config(self.h, None))
            return
        if isinstance(cfg, dict):
            c = DasConfig()
            for k, v in cfg.items():
                setattr(c, k, int(v))
            cfg = c
        check(load().ffdas_das_set_config(self.h, ctypes.byref(cfg)))

    def get_config(self) -> DasConfig:
        c = DasConfig()
        check(load().ffdas_das_get_config(self.h, ctypes.byref(c)))
        return c

    def last_kernel_info(self) -> dict:
        k = KernelInfo()
        check(load().ffdas_get_last_kernel_info(self.h, ctypes.byref(k)))
        return k.as_dict()

    def set_kernel_timing(self, enable: bool) -> None:
        check(load().ffdas_set_kernel_timing(self.h, int(bool(enable))))

    def last_kernel_ms(self) -> float:
        ms = ctypes.c_float()
        check(load().ffdas_get_last_kernel_time(self.h, ctypes.byref(ms)))
        return float(ms.value)

    def set_channel_scale(self, scale_ptr, count: int) -> None:
        """Per-channel scale applied by the ingest of the following calls (device pointer; None clears)."""
        check(load().ffdas_set_channel_scale(self.h, scale_ptr, int(count) if scale_ptr else 0))

    def set_gram_engine(self, engine: int) -> None:
        """truncate_rank's Gram engine: 0 auto, 1 FP32 FMA kernel, 2 tensor cores where the input qualifies."""
        check(load().ffdas_set_gram_engine(self.h, int(engine)))

    def set_pair_buffer(self, ptr, nbytes: int) -> None:
        """Caller-owned buffer for the pair rows of the next calls (None clears)."""
        check(load().ffdas_set_pair_buffer(self.h, ptr, int(nbytes) if ptr else 0))

    def last_kernel_units(self):
        """Units the last timed call's kernel evaluated, or None when it does not count them."""
        u = ctypes.c_longlong()
        rc = load().ffdas_get_last_kernel_units(self.h, ctypes.byref(u))
        if rc == Error.INVALID_STATE:
            return None
        check(rc)
        return int(u.value)

    def device_status(self) -> int:
        s = ctypes.c_int()
        check(load().ffdas_get_device_status(self.h, ctypes.byref(s)))
        return int(s.value)

    def measure_fp32_peak(self) -> float:
        tf = ctypes.c_double()
        check(load().ffdas_measure_fp32_peak(self.h, ctypes.byref(tf)))
        return float(tf.value)

    def destroy(self) -> None:
        if self.h:
            load().ffdas_destroy(self.h)
            self.h = c_handle()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def device_get() -> int:
    d = ctypes.c_int()
    check(load().ffdas_device_get(ctypes.byref(d)))
    return d.value


def device_set(device: int) -> None:
    check(load().ffdas_device_set(int(device)))


def device_count() -> int:
    d = ctypes.c_int()
    check(load().ffdas_device_count(ctypes.byref(d)))
    return d.value


def pair_bytes(desc: "TensorDesc", compute_type: int) -> int:
    """Bytes of a pair buffer for a forward call on x (ffdas_das_pair_bytes)."""
    n = ctypes.c_size_t()
    check(load().ffdas_das_pair_bytes(desc.desc, int(compute_type), ctypes.byref(n)))
    return int(n.value)


def event_create() -> int:
    e = ctypes.c_size_t()
    check(load().ffdas_event_create(ctypes.byref(e)))
    return int(e.value)


def event_destroy(e: int) -> None:
    check(load().ffdas_event_destroy(int(e)))


def event_record(handle: Handle, e: int) -> None:
    check(load().ffdas_event_record(handle.h, int(e)))


def event_synchronize(e: int) -> None:
    check(load().ffdas_event_synchronize(int(e)))


def event_elapsed_time(start: int, stop: int) -> float:
    ms = ctypes.c_float()
    check(load().ffdas_event_elapsed_time(int(start), int(stop), ctypes.byref(ms)))
    return float(ms.value)
