"""Per-device handle cache (reference: bindings/python/ffdas/_core/library.py:17-32).

One ffdas handle per CUDA device, created on first use and destroyed at exit.
Before returning a handle the library's current device is aligned with the
requested one, because the C entry points check it (DEVICE_MISMATCH).
"""
from __future__ import annotations

import atexit
import threading

import torch

from . import _lib

_handles: dict[int, _lib.Handle | None] = {}
_lock = threading.Lock()


def get_cuda_device() -> int:
    return _lib.device_get()


def set_cuda_device(device: int) -> None:
    _lib.device_set(device)


def get_library_handle(device=None) -> _lib.Handle:
    if device is None:
        index = torch.cuda.current_device()
    else:
        index = torch.device(device).index
        if index is None:
            index = torch.cuda.current_device()
    if _lib.device_get() != index:
        _lib.device_set(index)
    with _lock:
        h = _handles.get(index)
        if h is None:
            h = _lib.Handle()
            _handles[index] = h
    return h


@atexit.register
def _cleanup() -> None:
    for dev in list(_handles):
        h = _handles.get(dev)
        if h is not None:
            try:
                h.destroy()
            except Exception:
                pass
        _handles[dev] = None
