"""Device-side interval timer for delay-and-sum calls.

`Timer` keeps the public shape of the reference's timer
(bindings/python/ffdas/utils/timing.py: `Timer`, `start`, `stop`,
`elapsed_ms`, use as a context manager).  Its body is built on this library's
own event entry points (`ffdas_event_*`, recorded on the handle's stream after
pointing it at torch's current stream):

* the two events are created once per timer and released by a
  `weakref.finalize` hook, so they are freed when the timer is collected or at
  interpreter exit, whichever comes first, without a `__del__`;
* `stop()` only records; the host waits for the stop event when the interval
  is first read, so a timed block can be followed by more work before the
  result is needed;
* a timer can be restarted after a completed interval; the previous interval
  is then discarded.

    with Timer() as t:
        img = ffdas_b200.das(x, srcpos, dstpos, offsets, weights)
    print(t.elapsed_ms())
"""
from __future__ import annotations

import weakref

import torch

from . import _lib
from .library import get_library_handle


def _release(events: list) -> None:
    for e in events:
        try:
            _lib.event_destroy(e)
        except Exception:   # library already unloaded at interpreter exit
            pass
    events.clear()


class Timer:
    """Elapsed device time, in milliseconds, of the work enqueued on torch's
    current stream between `start()` and `stop()`."""

    _IDLE, _RUNNING, _RECORDED = 0, 1, 2

    def __init__(self, device=None):
        self._device = device
        self._handle = get_library_handle(device)
        self._events = [_lib.event_create(), _lib.event_create()]
        self._finalizer = weakref.finalize(self, _release, self._events)
        self._state = Timer._IDLE
        self._ms = None

    def _record(self, which: int) -> None:
        self._handle.set_stream(torch.cuda.current_stream(self._device).cuda_stream)
        _lib.event_record(self._handle, self._events[which])

    def start(self) -> None:
        if self._state == Timer._RUNNING:
            raise RuntimeError("Timer.start() called again before stop()")
        self._ms = None
        self._record(0)
        self._state = Timer._RUNNING

    def stop(self) -> None:
        if self._state != Timer._RUNNING:
            return
        self._record(1)
        self._state = Timer._RECORDED

    def elapsed_ms(self) -> float:
        if self._state != Timer._RECORDED:
            raise RuntimeError("Timer has no completed start()/stop() interval")
        if self._ms is None:
            _lib.event_synchronize(self._events[1])
            self._ms = _lib.event_elapsed_time(self._events[0], self._events[1])
        return self._ms

    def __enter__(self) -> "Timer":
        self.start()
        return self

    def __exit__(self, *exc) -> bool:
        self.stop()
        return False

    def close(self) -> None:
        """Release the two events now instead of at collection."""
        self._finalizer()
