"""Continuous-batching NUFFT server.

Requests (type 1, 2 or 3; 1D/2D/3D; any size) arrive at any time.  The server
admits pending requests as soon as stream slots are free and their device-memory
estimates fit the HBM budget (looking past a head request that does not fit, so
small requests are not blocked behind a large one).  Admitted small type-1/2
requests that share a dimension, precision and eps form a WAVE: one library call
(nfx_wave) enqueues all of them on one slot's stream with one persistent spread
launch over the bin tiles of every type-1 problem, one persistent interpolation
over those of every type-2 problem and one launch each for their deconvolution
passes.  Larger requests, type 3 and requests on shared points run alone on a
slot's stream.  Slots overlap on the device; completion is detected with CUDA
events and releases the slot and the memory.  Between requests the server keeps
on the device: cuFFT plans (library cache), fine-grid buffers (a pool per shape,
reused across requests) and sorted point sets (kept under a caller-chosen
`points_id` and reused by later requests on the same points, ordered after the
sort that produced them by an event).  Latency is measured from arrival to the
host seeing the completion event; `stats()` gives p50/p99 and throughput.
"""

from __future__ import annotations

import collections
import dataclasses
import math
import threading
import time
from typing import Callable, Optional, Sequence

import numpy as np
import torch

from ctypes import byref, c_size_t, c_void_p

from . import _lib
from ._plan import (PointSort, _facs, complex_dtype, deconv_pad, deconv_shuffle, fft_inplace, make_opts, precision_of,
                    ptr, real_dtype)
from .grid import compute_grid_size
from .kernel import compute_kernel_params
from .transforms import _fft_sign_type1, _fft_sign_type2, _type3_forward


_ITEMSIZE = {torch.complex64: 8, torch.complex128: 16}


@dataclasses.dataclass
class Request:
    """One transform.  kind: 1, 2 or 3.  For types 1/2 `n_modes` are the modes
    per axis; for type 3 `n_modes` is the type-3 grid (compute_type3_grid_size*).
    Inputs are device tensors, or `make_inputs(device, stream)` builds them at
    admission (returning the same fields)."""

    kind: int
    dim: int
    n_modes: tuple
    M: int
    K: int = 0
    coords: Optional[Sequence[torch.Tensor]] = None
    strengths: Optional[torch.Tensor] = None  # type 1/3: c (M,); type 2: f (modes)
    targets: Optional[Sequence[torch.Tensor]] = None  # type 3
    make_inputs: Optional[Callable] = None
    isign: Optional[int] = None
    eps: float = 1e-6
    dtype: torch.dtype = torch.complex64  # of inputs that make_inputs builds at admission
    points_id: Optional[object] = None
    arrival: float = 0.0
    # filled by the server
    result: Optional[torch.Tensor] = None
    error: Optional[str] = None  # set when the request could not run (it fails alone)
    admitted: float = 0.0
    finished: float = 0.0
    nbytes: int = 0

    def points(self) -> int:
        return self.M if self.kind != 3 else self.M + self.K


def estimate_bytes(req: Request) -> int:
    """Device bytes a request holds while in flight (inputs, outputs, sort
    workspace, fine grid(s) and cuFFT work area), complex64."""
    kp = compute_kernel_params(req.eps)
    pts = req.M
    inputs = pts * (4 * req.dim + 8)
    sort_ws = pts * (22 + 4 * req.dim) + 4 * 1024 * 1024  # sort tables + sorted folded coordinates
    if req.kind == 3:
        nf = [compute_grid_size(n, 2.0, kp.nspread) for n in req.n_modes]
        grid = 8 * math.prod(req.n_modes) + 2 * 8 * math.prod(nf)
        out = req.K * (8 + 4 * req.dim) * 2
        sort_ws += req.K * (22 + 4 * req.dim)
    else:
        nf = [compute_grid_size(n, 2.0, kp.nspread) for n in req.n_modes]
        grid = 2 * 8 * math.prod(nf)
        out = 8 * max(pts, math.prod(req.n_modes))
    return int(inputs + sort_ws + grid + out)


class _Slot:
    def __init__(self, device):
        self.stream = torch.cuda.Stream(device=device)
        self.reqs: list[Request] = []  # the request, or a wave's requests, in flight on this slot
        self.done = torch.cuda.Event()
        self.grids: list = []
        # sorted point sets and per-request buffers the work in flight reads:
        # kept alive until the slot's completion event, so an eviction from the
        # points cache (or a dropped reference) cannot free memory this slot's
        # stream still reads
        self.held: list = []
        self.ws: Optional[torch.Tensor] = None  # sort workspace, reused by the slot's next single request
        self.table: Optional[torch.Tensor] = None  # a wave's device problem table
        self.staging: Optional[torch.Tensor] = None  # its pinned host staging (untouched until done)

    def workspace(self, nbytes: int, device) -> torch.Tensor:
        if self.ws is None or self.ws.numel() < nbytes:
            self.ws = None
            self.ws = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
        return self.ws

    def wave_buffers(self, nbytes: int, device):
        if self.table is None or self.table.numel() < nbytes:
            n = max(nbytes, 64 << 10)
            self.table = torch.empty(n, dtype=torch.uint8, device=device)
            self.staging = torch.empty(n, dtype=torch.uint8).pin_memory()
        return self.table, self.staging


@dataclasses.dataclass
class _Shape:
    """Per-shape state of the one-call type 1/2 path: library options, fine grid,
    deconvolution factors (device) and the FFT sign."""

    opts: _lib.NfxOpts
    nf: tuple
    modes: object
    facs: list
    fac_ptrs: list
    sign: int


class NufftServer:
    """slots: concurrent requests (one CUDA stream each); hbm_budget: bytes of
    in-flight requests; keep_results=False drops each result once it is complete
    (throughput runs); pool_fraction of the budget may stay resident as pooled
    fine grids (least recently used shapes are dropped beyond it)."""

    def __init__(self, device=None, slots: int = 8, hbm_budget: float = 150e9, lookahead: int = 64,
                 keep_points: int = 64, keep_results: bool = True, pool_fraction: float = 0.1,
                 wave_max_points: int = 1 << 18, wave_size: int = 32):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.slots = [_Slot(self.device) for _ in range(slots)]
        self.budget = int(hbm_budget)
        self.in_use = 0
        self.lookahead = lookahead
        self.pending: collections.deque[Request] = collections.deque()
        self.completed: list[Request] = []
        self.grid_pool: "collections.OrderedDict[tuple, list[torch.Tensor]]" = collections.OrderedDict()
        self.pool_bytes = 0
        self.pool_cap = int(pool_fraction * hbm_budget)
        self.keep_results = keep_results
        self.points_cache: "collections.OrderedDict[object, tuple[PointSort, torch.cuda.Event]]" = \
            collections.OrderedDict()
        self.keep_points = keep_points
        self.shapes: "collections.OrderedDict[tuple, _Shape]" = collections.OrderedDict()
        # per-shape library options kept (least recently used out); the device
        # factors they point at stay alive in the library-wide factor cache
        self.keep_shapes = 4096
        # type-1/2 requests of at most wave_max_points points (without a
        # points_id) are grouped into waves of at most wave_size requests
        self.wave_max_points = wave_max_points
        self.wave_size = wave_size
        self.lock = threading.Lock()

    # -- resident state -----------------------------------------------------------
    @staticmethod
    def _size_class(nbytes: int) -> int:
        """Bytes of the pooled buffer that serves a request of nbytes: four
        classes per power of two (at most 25 % over), at least 1 MiB."""
        nbytes = max(int(nbytes), 1 << 20)
        step = 1 << max(nbytes.bit_length() - 3, 0)
        return -(-nbytes // step) * step

    def _flat(self, nbytes: int, slot: _Slot) -> torch.Tensor:
        """A device buffer of at least nbytes from the size-class pool (fine grids
        of every shape and wave workspaces share it), held by the slot until its
        work completes."""
        key = self._size_class(nbytes)
        pool = self.grid_pool.get(key)
        if pool:
            buf = pool.pop()
            self.pool_bytes -= buf.numel()
        else:
            buf = torch.empty(key, dtype=torch.uint8, device=self.device)
        slot.grids.append((key, buf))
        return buf

    def _grid(self, shape, dtype, slot: _Slot) -> torch.Tensor:
        nbytes = math.prod(shape) * _ITEMSIZE[dtype]
        return self._flat(nbytes, slot)[:nbytes].view(dtype).view(shape)

    def _return_grid(self, key, buf):
        self.grid_pool.setdefault(key, []).append(buf)
        self.grid_pool.move_to_end(key)
        self.pool_bytes += buf.numel()
        while self.pool_bytes > self.pool_cap and self.grid_pool:
            k, lst = next(iter(self.grid_pool.items()))
            while lst and self.pool_bytes > self.pool_cap:
                old = lst.pop()
                self.pool_bytes -= old.numel()
            if not lst:
                del self.grid_pool[k]

    def _sorted(self, req: Request, coords, nf, kp, slot: _Slot) -> PointSort:
        key = (req.points_id, tuple(nf), kp.nspread) if req.points_id is not None else None
        if key is not None and key in self.points_cache:
            ps, ev = self.points_cache[key]
            self.points_cache.move_to_end(key)
            slot.stream.wait_event(ev)
            slot.held.append(ps)
            return ps
        ps = PointSort(list(coords), nf, kp, prenorm=True)
        slot.held.append(ps)
        if key is not None:
            ev = torch.cuda.Event()
            ev.record(slot.stream)
            self.points_cache[key] = (ps, ev)
            while len(self.points_cache) > self.keep_points:
                self.points_cache.popitem(last=False)
        return ps

    def _shape(self, req: Request, precision: int) -> _Shape:
        key = (req.kind, tuple(req.n_modes), req.eps, req.isign, precision)
        sh = self.shapes.get(key)
        if sh is not None:
            self.shapes.move_to_end(key)
        else:
            kp = compute_kernel_params(req.eps)
            nf = tuple(compute_grid_size(n, 2.0, kp.nspread) for n in req.n_modes)
            facs = _facs(nf, req.n_modes, kp, precision, self.device)
            if req.kind == 1:
                sign = _fft_sign_type1(1 if req.isign is None else req.isign)
            else:
                sign = _fft_sign_type2(-1 if req.isign is None else req.isign)
            sh = _Shape(make_opts(precision, nf, kp, prenorm=True), nf, _lib.int3(req.n_modes), facs,
                        [ptr(f) for f in facs], sign)
            self.shapes[key] = sh
            while len(self.shapes) > self.keep_shapes:
                self.shapes.popitem(last=False)
        return sh

    def _run_one_call(self, req: Request, slot: _Slot):
        """Type 1/2 on unshared points: one library call (sort, spread or interp,
        FFT, deconvolution) on the slot's pooled workspace and a pooled grid."""
        c = req.strengths.contiguous()
        precision = precision_of(c.dtype)
        xs = [x.contiguous() for x in req.coords]
        if len(xs) != req.dim or any(x.dtype != real_dtype(precision) or x.shape != (req.M,) for x in xs):
            raise ValueError(f"coordinates must be {req.dim} tensors of shape ({req.M},), {real_dtype(precision)}")
        want = (req.M,) if req.kind == 1 else tuple(reversed(req.n_modes))
        if tuple(c.shape) != want:
            raise ValueError(f"type-{req.kind} strengths must have shape {want}")
        sh = self._shape(req, precision)
        lib = _lib.load()
        nbytes = c_size_t(0)
        _lib.check(lib.nfx_sort_workspace_bytes(byref(sh.opts), req.M, byref(nbytes)), "nfx_sort_workspace_bytes")
        ws = slot.workspace(int(nbytes.value), self.device)
        fw = self._grid((1,) + sh.nf[::-1], c.dtype, slot)
        xyz = [ptr(x) for x in xs] + [None] * (3 - len(xs))
        stream = c_void_p(slot.stream.cuda_stream)
        if req.kind == 1:
            out = torch.empty(tuple(reversed(req.n_modes)), dtype=complex_dtype(precision), device=self.device)
            _lib.check(lib.nfx_nufft1(byref(sh.opts), sh.modes, *xyz, req.M, ptr(c), 1, sh.sign, *sh.fac_ptrs,
                                      ptr(fw), ptr(out), ptr(ws), ws.numel(), stream), "nfx_nufft1")
        else:
            out = torch.empty(req.M, dtype=complex_dtype(precision), device=self.device)
            _lib.check(lib.nfx_nufft2(byref(sh.opts), sh.modes, *xyz, req.M, ptr(c), 1, sh.sign, *sh.fac_ptrs,
                                      ptr(fw), ptr(out), ptr(ws), ws.numel(), stream), "nfx_nufft2")
        req.result = out

    # -- execution ------------------------------------------------------------------
    def _run(self, req: Request, slot: _Slot):
        with torch.cuda.device(self.device), torch.cuda.stream(slot.stream):
            if req.make_inputs is not None:
                req.coords, req.strengths, req.targets = req.make_inputs(self.device)
            kp = compute_kernel_params(req.eps)
            if req.kind in (1, 2) and req.points_id is None:
                self._run_one_call(req, slot)
            elif req.kind == 1:
                isign = 1 if req.isign is None else req.isign
                nf = tuple(compute_grid_size(n, 2.0, kp.nspread) for n in req.n_modes)
                ps = self._sorted(req, req.coords, nf, kp, slot)
                fw = self._grid((1,) + nf[::-1], req.strengths.dtype, slot)
                ps.spread(req.strengths.reshape(1, -1), out=fw)
                fft_inplace(fw, req.dim, _fft_sign_type1(isign))
                req.result = deconv_shuffle(fw, req.n_modes, kp)[0]
            elif req.kind == 2:
                isign = -1 if req.isign is None else req.isign
                nf = tuple(compute_grid_size(n, 2.0, kp.nspread) for n in req.n_modes)
                fw = self._grid((1,) + nf[::-1], req.strengths.dtype, slot)
                deconv_pad(req.strengths.reshape((1,) + req.strengths.shape), nf, kp, out=fw)
                fft_inplace(fw, req.dim, _fft_sign_type2(isign))
                ps = self._sorted(req, req.coords, nf, kp, slot)
                req.result = ps.interp(fw)[0]
            else:
                isign = 1 if req.isign is None else req.isign
                req.result = _type3_forward(list(req.coords), req.strengths.reshape(1, -1), list(req.targets),
                                            tuple(req.n_modes), req.eps, isign, 2.0,
                                            ws_alloc=lambda n: slot.workspace(n, self.device))[0]
            slot.done.record(slot.stream)

    def _wave_key(self, req: Request):
        """Requests with the same key may share a wave (None: runs alone)."""
        if req.kind not in (1, 2) or req.points_id is not None or req.M > self.wave_max_points:
            return None
        dtype = req.strengths.dtype if req.strengths is not None else req.dtype
        return (req.dim, req.eps, dtype)

    def _wave_member(self, req: Request, slot: _Slot, lib):
        """Inputs, validation and buffers of one wave member; returns its item
        fields and library options (raises for a malformed request)."""
        if req.make_inputs is not None:
            req.coords, req.strengths, req.targets = req.make_inputs(self.device)
        c = req.strengths.contiguous()
        precision = precision_of(c.dtype)
        xs = [x.contiguous() for x in req.coords]
        if len(xs) != req.dim or any(x.dtype != real_dtype(precision) or x.shape != (req.M,) for x in xs):
            raise ValueError(f"coordinates must be {req.dim} tensors of shape ({req.M},), {real_dtype(precision)}")
        want = (req.M,) if req.kind == 1 else tuple(reversed(req.n_modes))
        if tuple(c.shape) != want:
            raise ValueError(f"type-{req.kind} strengths must have shape {want}")
        sh = self._shape(req, precision)
        nbytes = c_size_t(0)
        _lib.check(lib.nfx_sort_workspace_bytes(byref(sh.opts), req.M, byref(nbytes)), "nfx_sort_workspace_bytes")
        ws = self._flat(int(nbytes.value), slot)
        fw = self._grid((1,) + sh.nf[::-1], c.dtype, slot)
        shape = tuple(reversed(req.n_modes)) if req.kind == 1 else (req.M,)
        out = torch.empty(shape, dtype=complex_dtype(precision), device=self.device)
        slot.held += [xs, c, ws]
        return (xs, c, ws, fw, out, sh)

    def _run_wave(self, reqs: Sequence[Request], slot: _Slot):
        """A wave of small type-1/2 requests as one nfx_wave call on the slot's
        stream; a malformed member fails alone, the others run."""
        lib = _lib.load()
        with torch.cuda.device(self.device), torch.cuda.stream(slot.stream):
            members = []
            for req in reqs:
                try:
                    members.append((req, self._wave_member(req, slot, lib)))
                except (ValueError, TypeError, RuntimeError, NotImplementedError) as e:
                    req.error = f"{type(e).__name__}: {e}"
                    req.result = None
            if members:
                n = len(members)
                items = (_lib.NfxWaveItem * n)()
                for it, (req, (xs, c, ws, fw, out, sh)) in zip(items, members):
                    it.kind = req.kind
                    it.M = req.M
                    it.x, it.y, it.z = [x.data_ptr() for x in xs] + [None] * (3 - req.dim)
                    it.nf = _lib.int3(sh.nf)
                    it.n_modes = sh.modes
                    it.fft_sign = sh.sign
                    it.fac = (c_void_p * 3)(*[f.value if f is not None else None for f in sh.fac_ptrs])
                    it.in_ = c.data_ptr()
                    it.out = out.data_ptr()
                    it.fw = fw.data_ptr()
                    it.workspace = ws.data_ptr()
                    it.workspace_bytes = ws.numel()
                common = members[0][1][5].opts
                tb = c_size_t(0)
                _lib.check(lib.nfx_wave_table_bytes(byref(common), items, n, byref(tb)), "nfx_wave_table_bytes")
                table, staging = slot.wave_buffers(int(tb.value), self.device)
                try:
                    _lib.check(lib.nfx_wave(byref(common), items, n, ptr(table), ptr(staging), table.numel(),
                                            c_void_p(slot.stream.cuda_stream)), "nfx_wave")
                    for req, m in members:
                        req.result = m[4]
                except (ValueError, RuntimeError, NotImplementedError) as e:
                    for req, _ in members:
                        req.error = f"{type(e).__name__}: {e}"
                        req.result = None
            slot.done.record(slot.stream)

    def submit(self, req: Request):
        if req.arrival == 0.0:
            req.arrival = time.perf_counter()
        req.nbytes = estimate_bytes(req)
        with self.lock:
            self.pending.append(req)

    def _admit(self):
        free = [s for s in self.slots if not s.reqs]
        if not free:
            return
        with self.lock:
            # choose, in arrival order within the lookahead, the requests that fit
            # the budget and a slot.  Small requests spread over the free slots
            # first (a wave of one runs alone); only a backlog of more small
            # requests than free slots is packed, up to wave_size per wave
            look = min(self.lookahead, len(self.pending))
            n_small = sum(1 for k in range(look) if self._wave_key(self.pending[k]) is not None)
            cap = min(self.wave_size, max(1, -(-n_small // len(free))))
            singles: list[Request] = []
            waves: list[list[Request]] = []
            open_wave: dict = {}
            i = 0
            while i < min(self.lookahead, len(self.pending)):
                req = self.pending[i]
                if not (self.in_use + req.nbytes <= self.budget or self.in_use == 0):
                    i += 1
                    continue
                key = self._wave_key(req)
                joins = key is not None and key in open_wave and len(open_wave[key]) < cap
                if not joins and len(singles) + len(waves) >= len(free):
                    i += 1
                    continue
                del self.pending[i]
                self.in_use += req.nbytes
                req.admitted = time.perf_counter()
                if key is None:
                    singles.append(req)
                elif joins:
                    open_wave[key].append(req)
                else:
                    open_wave[key] = [req]
                    waves.append(open_wave[key])
        for group in [[r] for r in singles] + waves:
            slot = free.pop()
            slot.reqs = list(group)
            try:
                if len(group) == 1:
                    self._run(group[0], slot)
                else:
                    self._run_wave(group, slot)
            except (ValueError, TypeError, RuntimeError, NotImplementedError) as e:
                # a malformed request fails alone (a wave fails as a whole); the
                # slot is released by the normal completion path once its stream
                # is idle
                for req in group:
                    req.error = f"{type(e).__name__}: {e}"
                    req.result = None
                slot.done.record(slot.stream)

    def _poll(self):
        for s in self.slots:
            if s.reqs and s.done.query():
                now = time.perf_counter()
                for key, g in s.grids:
                    self._return_grid(key, g)
                s.grids = []
                s.held = []
                for req in s.reqs:
                    req.finished = now
                    self.in_use -= req.nbytes
                    if req.make_inputs is not None:  # inputs were generated here: release them
                        req.coords = req.strengths = req.targets = None
                    if not self.keep_results:
                        req.result = None
                    self.completed.append(req)
                s.reqs = []

    def busy(self) -> bool:
        return bool(self.pending) or any(s.reqs for s in self.slots)

    def step(self):
        self._poll()
        self._admit()

    def serve(self, requests: Sequence[Request], arrivals: Sequence[float] | None = None, idle_sleep: float = 2e-5):
        """Feed requests at their arrival offsets (seconds from now) and run
        until all complete.  Returns the completed requests."""
        t0 = time.perf_counter()
        arrivals = arrivals if arrivals is not None else [0.0] * len(requests)
        order = sorted(range(len(requests)), key=lambda i: arrivals[i])
        nxt = 0
        while nxt < len(order) or self.busy():
            now = time.perf_counter()
            while nxt < len(order) and t0 + arrivals[order[nxt]] <= now:
                r = requests[order[nxt]]
                r.arrival = t0 + arrivals[order[nxt]]
                self.submit(r)
                nxt += 1
            self.step()
            if nxt < len(order) and not self.pending:
                wait = t0 + arrivals[order[nxt]] - time.perf_counter()
                if wait > 0:
                    time.sleep(min(wait, 1e-3))
            elif self.busy():
                time.sleep(idle_sleep)
        return self.completed

    def stats(self, reqs: Sequence[Request] | None = None) -> dict:
        """p50 / p99 / mean latency and throughput over the requests that ran."""
        reqs = [r for r in (reqs if reqs is not None else self.completed) if r.error is None]
        lat = np.array([r.finished - r.arrival for r in reqs]) * 1e3
        pts = sum(r.points() for r in reqs)
        span = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
        return {"requests": len(reqs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "points": int(pts), "points_per_s": pts / span, "span_s": span}
