"""CUDA-event timer on the library handle's stream (reference: bindings/python/ffdas/utils/timing.py:5)."""
from __future__ import annotations

import torch

from . import _lib
from .library import get_library_handle


class Timer:
    """Context manager recording ffdas events around a block of GPU work.

    The handle's stream is set to torch's current stream first, so the events
    bracket the work that `das` enqueues.

        with Timer() as t:
            img = ffdas_b200.das(x, srcpos, dstpos, offsets, weights)
        print(t.elapsed_ms())
    """

    def __init__(self, device=None):
        self._handle = get_library_handle(device)
        self._device = device
        self._start = _lib.event_create()
        self._stop = _lib.event_create()
        self._running = False
        self._elapsed = None

    def start(self):
        if self._running:
            raise RuntimeError("Timer is already running")
        self._handle.set_stream(torch.cuda.current_stream(self._device).cuda_stream)
        self._running = True
        _lib.event_record(self._handle, self._start)

    def stop(self):
        if not self._running:
            return
        self._handle.set_stream(torch.cuda.current_stream(self._device).cuda_stream)
        _lib.event_record(self._handle, self._stop)
        _lib.event_synchronize(self._stop)
        self._elapsed = _lib.event_elapsed_time(self._start, self._stop)
        self._running = False

    def __enter__(self):
        self.start()
        return self

    def __exit__(self, *exc):
        self.stop()
        return False

    def elapsed_ms(self) -> float:
        if self._elapsed is None:
            raise RuntimeError("Timer has not been stopped yet")
        return self._elapsed

    def __del__(self):
        try:
            if self._start:
                _lib.event_destroy(self._start)
                self._start = 0
            if self._stop:
                _lib.event_destroy(self._stop)
                self._stop = 0
        except Exception:
            pass
