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
def record():
    rec = Recorder()
    prev = getattr(_state, "rec", None)
    _state.rec = rec
    try:
        yield rec
    finally:
        _state.rec = prev


@contextlib.contextmanager
def span(name: str, device, launches: int | None = None):
    rec = getattr(_state, "rec", None)
    if rec is None:
        yield
        return
    stream = torch.cuda.current_stream(device)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    try:
        yield
    finally:
        b.record(stream)
        rec.events.append((name, a, b, LAUNCHES.get(name, 1) if launches is None else launches))
