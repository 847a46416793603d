"""Device plumbing: sorted point sets and calls into libnfx_b200.

A `PointSort` owns the workspace of one bin sort (coordinates + grid + kernel)
and runs spread / interp / gradient passes against it.  torch supplies device
memory and the current stream; all arithmetic happens in the CUDA library.
"""

from __future__ import annotations

import collections
import threading
import ctypes
from ctypes import byref, c_int, c_size_t, c_void_p
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .kernel import KernelParams, deconv_factors
from .profiling import span

_REAL = {_lib.NFX_F32: torch.float32, _lib.NFX_F64: torch.float64}
_CPLX = {_lib.NFX_F32: torch.complex64, _lib.NFX_F64: torch.complex128}


def precision_of(dtype: torch.dtype) -> int:
    if dtype in (torch.complex64, torch.float32):
        return _lib.NFX_F32
    if dtype in (torch.complex128, torch.float64):
        return _lib.NFX_F64
    raise TypeError(f"unsupported dtype {dtype}; use complex64/float32 or complex128/float64")


def real_dtype(precision: int) -> torch.dtype:
    return _REAL[precision]


def complex_dtype(precision: int) -> torch.dtype:
    return _CPLX[precision]


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def stream_of(device: torch.device) -> int:
    """Handle of the current stream of `device` (the raw query when torch has it:
    no Stream object per call)."""
    if _raw_stream is not None:
        return _raw_stream(device.index if device.index is not None else torch.cuda.current_device())
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t: torch.Tensor | None):
    return None if t is None else c_void_p(t.data_ptr())


def require_cuda(t: torch.Tensor, what: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{what} must be a CUDA tensor")


_opts_cache: dict = {}
_opts_lock = threading.Lock()


def make_opts(precision: int, nf: Sequence[int], kp: KernelParams, prenorm: bool, tile=None,
              max_subproblem: int = 0, modes=(0, 0)) -> _lib.NfxOpts:
    """Library options with default tiles filled in; a private copy of a cached
    struct per (precision, grid, kernel, tiling, threads-per-point modes) key.
    modes = (spread_mode, interp_mode), NFX_PER_POINT_* (0: the library's choice)."""
    key = (precision, tuple(int(n) for n in nf), int(kp.nspread), float(kp.beta), float(kp.c), bool(prenorm),
           None if tile is None else tuple(int(t) for t in tile), int(max_subproblem), tuple(modes))
    with _opts_lock:
        o = _opts_cache.get(key)
    if o is None:
        o = _make_opts(precision, nf, kp, prenorm, tile, max_subproblem, modes)
        with _opts_lock:
            if len(_opts_cache) >= 4096:
                _opts_cache.clear()
            _opts_cache[key] = o
    return _lib.NfxOpts.from_buffer_copy(o)


def _make_opts(precision: int, nf: Sequence[int], kp: KernelParams, prenorm: bool, tile,
               max_subproblem: int, modes=(0, 0)) -> _lib.NfxOpts:
    o = _lib.NfxOpts()
    o.precision = precision
    o.dim = len(nf)
    o.nf = _lib.int3(nf)
    o.nspread = int(kp.nspread)
    o.beta = float(kp.beta)
    o.kc = float(kp.c)
    o.prenorm = 1 if prenorm else 0
    o.tile = (c_int * 3)(0, 0, 0) if tile is None else _lib.int3(tile)
    o.max_subproblem = int(max_subproblem)
    o.spread_mode, o.interp_mode = (int(m) for m in modes)
    lib = _lib.load()
    _lib.check(lib.nfx_default_tiles(byref(o)), "nfx_default_tiles")
    return o


def sort_launches(opts, M: int, type3: bool = False) -> int:
    """Kernels one nfx_sort_points call launches (the library's own count for
    these options, M and point kind): keys with the first digit's counts, per
    radix pass a column scan and a scatter (plus a count for the passes after
    the first), the sorted-coordinates gather (double and type-3 points only),
    bin bounds (unless the last pass writes them) and subproblems."""
    n = c_int(0)
    _lib.check(_lib.load().nfx_sort_kernel_count(byref(opts), int(M), int(bool(type3)), byref(n)),
               "nfx_sort_kernel_count")
    return int(n.value)


class PointSort:
    """Bin-sorted non-uniform points on one fine grid."""

    def __init__(self, coords: Sequence[torch.Tensor], nf: Sequence[int], kp: KernelParams, prenorm: bool,
                 tile=None, max_subproblem: int = 0, modes=(0, 0)):
        self.dim = len(coords)
        if self.dim not in (1, 2, 3) or len(nf) != self.dim:
            raise ValueError("coords and nf must have 1, 2 or 3 axes")
        self.device = coords[0].device
        self.precision = precision_of(coords[0].dtype)
        self.coords = [c.contiguous() for c in coords]
        self.M = int(self.coords[0].shape[0])
        for c in self.coords:
            require_cuda(c, "coordinates")
            if c.dtype != self.coords[0].dtype or c.ndim != 1 or c.shape[0] != self.M:
                raise ValueError("coordinates must be 1D tensors of equal length and dtype")
        self.nf = tuple(int(n) for n in nf)
        self.kp = kp
        self.prenorm = prenorm
        self.opts = make_opts(self.precision, self.nf, kp, prenorm, tile, max_subproblem, modes)
        lib = _lib.load()
        nbytes = c_size_t(0)
        _lib.check(lib.nfx_sort_workspace_bytes(byref(self.opts), self.M, byref(nbytes)), "nfx_sort_workspace_bytes")
        self.ws_bytes = int(nbytes.value)
        self.ws = torch.empty(max(self.ws_bytes, 1), dtype=torch.uint8, device=self.device)
        self.stream = stream_of(self.device)  # the stream the sort ran on (and the workspace belongs to)
        self._src = None
        launches = lambda: sort_launches(self.opts, self.M)  # noqa: E731 (evaluated only when recording)
        with torch.cuda.device(self.device), span("nfx_sort_points", self.device, launches):
            _lib.check(lib.nfx_sort_points(byref(self.opts), *self._xyz(), self.M, ptr(self.ws), self.ws_bytes,
                                           c_void_p(stream_of(self.device))), "nfx_sort_points")
            # marks the sort's completion on its stream: a user on another stream
            # waits for it (sort_cache does that)
            self.ready = torch.cuda.Event()
            self.ready.record(torch.cuda.current_stream(self.device))

    # -- helpers -----------------------------------------------------------
    def _xyz(self):
        cs = [ptr(c) for c in self.coords] + [None] * (3 - self.dim)
        return cs[0], cs[1], cs[2]

    @property
    def grid_shape(self) -> tuple[int, ...]:
        return tuple(reversed(self.nf))

    @property
    def tile(self) -> tuple[int, ...]:
        return tuple(self.opts.tile[d] for d in range(self.dim))

    def _call(self, name: str, *args):
        lib = _lib.load()
        with torch.cuda.device(self.device), span(name, self.device, 1 if self.M > 0 else 0):
            _lib.check(getattr(lib, name)(byref(self.opts), *self._xyz(), self.M, *args, ptr(self.ws), self.ws_bytes,
                                          c_void_p(stream_of(self.device))), name)

    def results(self):
        """(keys, perm, bin_start) as int32 device tensors (for inspection and tests)."""
        lib = _lib.load()
        nb = c_int(0)
        _lib.check(lib.nfx_sort_results(byref(self.opts), self.M, ptr(self.ws), self.ws_bytes, None, None, None,
                                        byref(nb), None), "nfx_sort_results")
        keys = torch.empty(self.M, dtype=torch.int32, device=self.device)
        perm = torch.empty(self.M, dtype=torch.int32, device=self.device)
        bstart = torch.empty(nb.value + 1, dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(lib.nfx_sort_results(byref(self.opts), self.M, ptr(self.ws), self.ws_bytes, ptr(keys),
                                            ptr(perm), ptr(bstart), byref(nb), c_void_p(stream_of(self.device))),
                       "nfx_sort_results")
        return keys, perm, bstart

    def _check_strengths(self, c: torch.Tensor) -> torch.Tensor:
        if c.dtype != complex_dtype(self.precision) or c.shape[-1] != self.M or c.ndim != 2:
            raise ValueError(f"strengths must be (n_trans, {self.M}) {complex_dtype(self.precision)}")
        require_cuda(c, "strengths")
        return c.contiguous()

    def _check_grid(self, fw: torch.Tensor) -> torch.Tensor:
        if fw.dtype != complex_dtype(self.precision) or tuple(fw.shape[1:]) != self.grid_shape:
            raise ValueError(f"grid must be (n_trans, {self.grid_shape}) {complex_dtype(self.precision)}")
        require_cuda(fw, "grid")
        return fw.contiguous()

    # -- passes ------------------------------------------------------------
    def spread(self, c: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """c: (n_trans, M) -> fine grid (n_trans, nf_d, ..., nf_1)."""
        c = self._check_strengths(c)
        nt = c.shape[0]
        fw = out if out is not None else torch.empty((nt,) + self.grid_shape, dtype=c.dtype, device=self.device)
        self._call("nfx_spread_sorted", ptr(c), nt, ptr(fw))
        return fw

    def interp(self, fw: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """fine grid (n_trans, nf_d..nf_1) -> (n_trans, M)."""
        fw = self._check_grid(fw)
        nt = fw.shape[0]
        c = out if out is not None else torch.empty((nt, self.M), dtype=fw.dtype, device=self.device)
        self._call("nfx_interp_sorted", ptr(fw), nt, ptr(c))
        return c

    def spread_grad(self, c: torch.Tensor, g: torch.Tensor, need_c: bool, need_x: Sequence[bool]):
        """Backward of spread: (dc or None, [d_axis or None])."""
        c = self._check_strengths(c)
        g = self._check_grid(g)
        nt = c.shape[0]
        dc = torch.empty((nt, self.M), dtype=c.dtype, device=self.device) if need_c else None
        dxs = [torch.empty(self.M, dtype=real_dtype(self.precision), device=self.device) if (
            d < len(need_x) and need_x[d]) else None for d in range(self.dim)]
        outs = dxs + [None] * (3 - self.dim)
        self._call("nfx_spread_grad_sorted", ptr(c), ptr(g), nt, ptr(dc), ptr(outs[0]), ptr(outs[1]), ptr(outs[2]))
        return dc, dxs

    def interp_grad(self, fw: torch.Tensor, g: torch.Tensor, need_x: Sequence[bool]):
        """Coordinate part of the backward of interp: [d_axis or None]."""
        fw = self._check_grid(fw)
        g = self._check_strengths(g)
        nt = g.shape[0]
        dxs = [torch.empty(self.M, dtype=real_dtype(self.precision), device=self.device) if (
            d < len(need_x) and need_x[d]) else None for d in range(self.dim)]
        outs = dxs + [None] * (3 - self.dim)
        self._call("nfx_interp_grad_sorted", ptr(fw), ptr(g), nt, ptr(outs[0]), ptr(outs[1]), ptr(outs[2]))
        return dxs


# ---------------------------------------------------------------------------
# Caches: sorted point sets (keyed on live coordinate tensors) and factors.
# ---------------------------------------------------------------------------
class _SortCache:
    """LRU of PointSorts.  Entries hold strong references to their coordinate
    tensors, so a key (tensor identity, data pointer, version counter) can only
    match the same tensors unmodified through torch.

    A write that bypasses torch's version counter (a raw kernel, a ctypes or
    DLPack writer from another framework into the same memory) cannot be seen
    here: after one, call `invalidate(tensor)` (or `clear()`), or the next
    transform on those coordinates reuses the old sort and drops every point
    that left its tile.

    A cached sort may be used from another stream than the one that made it:
    that stream first waits for the sort's completion event, and the workspace
    is recorded on it, so an eviction cannot hand the memory to new work while
    the other stream's kernels still read it.

    During a CUDA graph capture a sort has only been captured, not run: it
    belongs to the graph and never enters this cache.  It is reused only by
    later transforms of the same capture (keyed by the capture's id), e.g. a
    type 2 after a type 1 on the same points, on another stream of the capture
    through the same event wait (a dependency inside the graph)."""

    def __init__(self, size: int = 4):
        self.size = size
        self.enabled = True
        self._d: "collections.OrderedDict[tuple, PointSort]" = collections.OrderedDict()
        self._cap: "collections.OrderedDict[tuple, PointSort]" = collections.OrderedDict()
        self._lock = threading.Lock()

    def _get_captured(self, coords, nf, kp, prenorm, key) -> PointSort:
        dev = coords[0].device
        s = stream_of(dev)
        cid = ctypes.c_ulonglong(0)
        _lib.check(_lib.load().nfx_capture_id(c_void_p(s), byref(cid)), "nfx_capture_id")
        ckey = (int(cid.value),) + key
        with self._lock:
            hit = self._cap.get(ckey)
        if hit is not None and all(a is b for a, b in zip(hit._src, coords)):
            if hit.stream != s:
                torch.cuda.current_stream(dev).wait_event(hit.ready)
            return hit
        ps = PointSort(coords, nf, kp, prenorm)
        ps._src = list(coords)
        with self._lock:
            self._cap[ckey] = ps
            while len(self._cap) > 2 * self.size:
                self._cap.popitem(last=False)
        return ps

    def get(self, coords, nf, kp, prenorm) -> PointSort:
        key = tuple((id(c), c.data_ptr(), c._version, c.dtype, c.shape[0]) for c in coords) + (
            tuple(nf), kp.nspread, float(kp.beta), float(kp.c), bool(prenorm))
        if torch.cuda.is_current_stream_capturing():
            return self._get_captured(coords, nf, kp, prenorm, key)
        if self.enabled:
            with self._lock:
                hit = self._d.get(key)
                if hit is not None and not all(a is b for a, b in zip(hit._src, coords)):
                    hit = None
                if hit is not None:
                    self._d.move_to_end(key)
            if hit is not None:
                s = stream_of(hit.device)
                if s != hit.stream:
                    cur = torch.cuda.ExternalStream(s, device=hit.device)
                    cur.wait_event(hit.ready)
                    hit.ws.record_stream(cur)
                return hit
        ps = PointSort(coords, nf, kp, prenorm)
        ps._src = list(coords)
        if self.enabled:
            with self._lock:
                self._d[key] = ps
                while len(self._d) > self.size:
                    self._d.popitem(last=False)
        return ps

    def invalidate(self, *tensors: torch.Tensor) -> int:
        """Drop every cached sort made from any of `tensors` (coordinates whose
        memory was written outside torch); returns the number dropped."""
        ptrs = {t.data_ptr() for t in tensors}
        with self._lock:
            dead = [k for k, ps in self._d.items() if any(c.data_ptr() in ptrs for c in ps._src)]
            for k in dead:
                del self._d[k]
        return len(dead)

    def clear(self):
        with self._lock:
            self._d.clear()
            self._cap.clear()


sort_cache = _SortCache()
_fac_cache: dict = {}
_fac_lock = threading.Lock()


def factors(nf: int, n_modes: int, kp: KernelParams, precision: int, device: torch.device) -> torch.Tensor:
    """Device copy of the per-axis deconvolution factors (cached)."""
    key = (nf, n_modes, kp.nspread, float(kp.beta), float(kp.c), precision, str(device))
    with _fac_lock:
        t = _fac_cache.get(key)
    if t is None:
        arr = deconv_factors(nf, n_modes, kp)
        t = torch.from_numpy(arr.astype(np.float32 if precision == _lib.NFX_F32 else np.float64)).to(device)
        with _fac_lock:
            # never evicted while the process runs: an enqueued deconvolution may
            # still read a factor tensor after its call returns (a few KB a shape)
            _fac_cache[key] = t
    return t


def clear_caches() -> None:
    """Drop cached point sorts, deconvolution factors and cuFFT plans.

    Enqueued deconvolutions (a server's requests in flight, work on any stream)
    may still read the factor tensors, so every device that holds one is
    synchronised before they are dropped."""
    sort_cache.clear()
    with _fac_lock:
        devs = {t.device for t in _fac_cache.values()}
        for d in devs:
            torch.cuda.synchronize(d)
        _fac_cache.clear()
    _lib.load().nfx_fft_cache_clear()


# ---------------------------------------------------------------------------
# Grid passes: FFT and deconvolution.
# ---------------------------------------------------------------------------
def fft_inplace(fw: torch.Tensor, dim: int, sign: int) -> torch.Tensor:
    """In-place batched FFT over the last `dim` axes of (n_trans, ...) grid."""
    precision = precision_of(fw.dtype)
    nf = tuple(reversed(fw.shape[-dim:]))
    lib = _lib.load()
    with torch.cuda.device(fw.device), span("nfx_fft", fw.device, 0):
        if torch.cuda.is_current_stream_capturing():
            # a captured FFT keeps its work area: take one from the graph's pool
            nbytes = c_size_t(0)
            _lib.check(lib.nfx_fft_work_bytes(precision, dim, _lib.int3c(nf), int(fw.shape[0]), byref(nbytes)),
                       "nfx_fft_work_bytes")
            work = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=fw.device)
            _lib.check(lib.nfx_fft_ws(precision, dim, _lib.int3c(nf), int(fw.shape[0]), ptr(fw), int(sign), ptr(work),
                                      work.numel(), c_void_p(stream_of(fw.device))), "nfx_fft_ws")
        else:
            _lib.check(lib.nfx_fft(precision, dim, _lib.int3c(nf), int(fw.shape[0]), ptr(fw), int(sign),
                                   c_void_p(stream_of(fw.device))), "nfx_fft")
    return fw


def _facs(nf, n_modes, kp, precision, device):
    fs = [factors(nf[d], n_modes[d], kp, precision, device) for d in range(len(nf))]
    return fs + [None] * (3 - len(fs))


def deconv_shuffle(fw_hat: torch.Tensor, n_modes: Sequence[int], kp: KernelParams) -> torch.Tensor:
    """(n_trans, nf_d..nf_1) FFT output -> (n_trans, n_d..n_1) CMCL modes."""
    dim = len(n_modes)
    precision = precision_of(fw_hat.dtype)
    nf = tuple(reversed(fw_hat.shape[-dim:]))
    fs = _facs(nf, n_modes, kp, precision, fw_hat.device)
    out = torch.empty((fw_hat.shape[0],) + tuple(reversed(n_modes)), dtype=fw_hat.dtype, device=fw_hat.device)
    lib = _lib.load()
    with torch.cuda.device(fw_hat.device), span("nfx_deconv_shuffle", fw_hat.device):
        _lib.check(lib.nfx_deconv_shuffle(precision, dim, _lib.int3c(nf), _lib.int3c(n_modes), ptr(fs[0]), ptr(fs[1]),
                                          ptr(fs[2]), ptr(fw_hat), ptr(out), int(fw_hat.shape[0]),
                                          c_void_p(stream_of(fw_hat.device))), "nfx_deconv_shuffle")
    return out


def deconv_pad(f: torch.Tensor, nf: Sequence[int], kp: KernelParams, out: torch.Tensor | None = None) -> torch.Tensor:
    """(n_trans, n_d..n_1) CMCL modes -> zero-padded deconvolved (n_trans, nf_d..nf_1)."""
    dim = len(nf)
    precision = precision_of(f.dtype)
    f = f.contiguous()
    n_modes = tuple(reversed(f.shape[-dim:]))
    fs = _facs(nf, n_modes, kp, precision, f.device)
    if out is None:
        out = torch.empty((f.shape[0],) + tuple(reversed(nf)), dtype=f.dtype, device=f.device)
    lib = _lib.load()
    with torch.cuda.device(f.device), span("nfx_deconv_pad", f.device):
        _lib.check(lib.nfx_deconv_pad(precision, dim, _lib.int3c(nf), _lib.int3c(n_modes), ptr(fs[0]), ptr(fs[1]),
                                      ptr(fs[2]), ptr(f), ptr(out), int(f.shape[0]), c_void_p(stream_of(f.device))),
                   "nfx_deconv_pad")
    return out
