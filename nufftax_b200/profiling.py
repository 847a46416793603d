"""Per-call CUDA-event timing of libnfx_b200 calls.

Inside `with record() as rec:`, every library call issued through the host
layer is bracketed by two CUDA events on the stream it is launched on, tagged
with the call name and the number of kernels it launches.  `rec.summary()`
gives per-name launch counts and device milliseconds (after a synchronize).
"""

from __future__ import annotations

import contextlib
import threading
from collections import defaultdict

import torch

_state = threading.local()

# kernels launched by one call of each library entry point
LAUNCHES = {"nfx_sort_points": 8, "nfx_spread_sorted": 1, "nfx_interp_sorted": 1, "nfx_spread_grad_sorted": 1,
            "nfx_interp_grad_sorted": 1, "nfx_deconv_shuffle": 1, "nfx_deconv_pad": 1, "nfx_t3_prepare": 0,
            "nfx_t3_finish": 1, "nfx_fft": 0}


class Recorder:
    def __init__(self):
        self.events = []
        self.only = None

    def summary(self):
        torch.cuda.synchronize()
        out = defaultdict(lambda: {"calls": 0, "ms": 0.0, "launches": 0})
        for name, a, b, n in self.events:
            s = out[name]
            s["calls"] += 1
            s["ms"] += a.elapsed_time(b)
            s["launches"] += n
        return dict(out)


@contextlib.contextmanager
def record(only=None):
    """Record the library calls of this thread (only those named in `only`, if
    given: fewer events on the host)."""
    rec = Recorder()
    rec.only = None if only is None else frozenset(only)
    prev = getattr(_state, "rec", None)
    _state.rec = rec
    try:
        yield rec
    finally:
        _state.rec = prev


class span:
    """Brackets one library call with CUDA events while a `record()` is active
    on this thread; otherwise does nothing (a plain object, no generator, so
    the common case costs a thread-local read).  `launches` (kernels the call
    launches) may be a callable, evaluated only when recording."""

    __slots__ = ("rec", "name", "stream", "launches", "a", "ext")

    def __init__(self, name: str, device, launches: int | None = None):
        self.rec = getattr(_state, "rec", None)
        if self.rec is not None and self.rec.only is not None and name not in self.rec.only:
            self.rec = None
        if self.rec is not None:
            self.name = name
            self.stream = torch.cuda.current_stream(device)
            if callable(launches):  # computed only when recording
                launches = launches()
            self.launches = LAUNCHES.get(name, 1) if launches is None else launches

    def __enter__(self):
        if self.rec is not None:
            # under CUDA graph capture the events become event-record nodes of
            # the graph (re-recorded by every replay)
            self.ext = torch.cuda.is_current_stream_capturing()
            self.a = torch.cuda.Event(enable_timing=True, external=self.ext)
            self.a.record(self.stream)
        return self

    def __exit__(self, *exc):
        if self.rec is not None:
            b = torch.cuda.Event(enable_timing=True, external=self.ext)
            b.record(self.stream)
            self.rec.events.append((self.name, self.a, b, self.launches))
        return False
