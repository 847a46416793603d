"""Batched NUFFTs: many independent problems of uneven size in one graph.

A `BatchPlan` holds P problems (own points, mode counts and tiling; shared eps,
precision and dimension).  One `run()` performs, for every problem, a type-1
transform of its strengths and a type-2 transform of its modes, as

    type 1: per-problem bin sorts (concurrent, on side streams) -> ONE
    persistent spread launch over the work queue of all problems' bin tiles ->
    one batched cuFFT per grid-size class -> ONE deconvolve/crop launch;
    type 2: ONE deconvolve/pad launch -> batched cuFFT (both while the points
    sort) -> ONE persistent interp launch once the sorts are done,

the two chains on their own streams and fine grids, so that they overlap,
captured once in a CUDA graph and replayed (`graph=True`).  The plan owns its
input and output buffers (`c_in`, `f_in`, `f_out`, `c_out`); callers write
inputs in place (or pass them to `run`) and read outputs after it.  Coordinates
are read at every run, so they may be updated in place between runs.
"""

from __future__ import annotations

import ctypes
from ctypes import byref, c_int, c_int64, c_size_t, c_void_p
from typing import Sequence

import torch

from . import _lib
from ._plan import complex_dtype, factors, precision_of, ptr, real_dtype, stream_of
from .grid import compute_grid_size
from .kernel import compute_kernel_params


def _fft_sign_type1(isign: int) -> int:
    return 1 if isign > 0 else -1


def _fft_sign_type2(isign: int) -> int:
    return -1 if isign < 0 else 1


class BatchPlan:
    def __init__(self, points: Sequence[Sequence[torch.Tensor]], n_modes: Sequence[Sequence[int]], eps: float = 1e-6,
                 isign_type1: int = 1, isign_type2: int = -1, upsampfac: float = 2.0,
                 dtype: torch.dtype = torch.complex64, tiles=None, max_subproblem=None, interp_modes=None,
                 graph: bool = True):
        if len(points) == 0 or len(points) != len(n_modes):
            raise ValueError("need one n_modes entry per problem")
        self.P = len(points)
        self.dim = len(points[0])
        self.device = points[0][0].device
        self.precision = precision_of(dtype)
        self.cdt = complex_dtype(self.precision)
        self.rdt = real_dtype(self.precision)
        self.eps = eps
        self.isign1, self.isign2 = int(isign_type1), int(isign_type2)
        self.kp = compute_kernel_params(eps, upsampfac)
        self.points = [[c.to(self.rdt).contiguous() for c in pts] for pts in points]
        for pts in self.points:
            if len(pts) != self.dim or any(not c.is_cuda for c in pts):
                raise ValueError("every problem needs dim CUDA coordinate tensors")
        self.M = [int(pts[0].shape[0]) for pts in self.points]
        self.n_modes = [tuple(int(v) for v in nm) for nm in n_modes]
        self.nf = [tuple(compute_grid_size(n, upsampfac, self.kp.nspread) for n in nm) for nm in self.n_modes]
        tiles = tiles if tiles is not None else [None] * self.P
        maxsub = max_subproblem if max_subproblem is not None else [0] * self.P
        imodes = interp_modes if interp_modes is not None else [0] * self.P
        self.lib = _lib.load()
        dev = self.device

        # buffers
        self.c_in = [torch.zeros(m, dtype=self.cdt, device=dev) for m in self.M]
        self.f_in = [torch.zeros(tuple(reversed(nm)), dtype=self.cdt, device=dev) for nm in self.n_modes]
        self.f_out = [torch.empty(tuple(reversed(nm)), dtype=self.cdt, device=dev) for nm in self.n_modes]
        self.c_out = [torch.empty(m, dtype=self.cdt, device=dev) for m in self.M]
        # fine grids grouped by shape (contiguous per group -> one batched FFT
        # each): one set for the type 1 (fw), one for the type 2 (fw2), so the
        # two chains do not wait for each other
        groups: dict[tuple, list[int]] = {}
        for p, nf in enumerate(self.nf):
            groups.setdefault(nf, []).append(p)

        def grid_set():
            gs, views = [], [None] * self.P
            for nf, members in groups.items():
                buf = torch.empty((len(members),) + tuple(reversed(nf)), dtype=self.cdt, device=dev)
                gs.append((nf, buf))
                for i, p in enumerate(members):
                    views[p] = buf[i]
            # cuFFT work areas owned by the plan (the captured graph keeps their
            # addresses), one per group: the groups' FFTs run concurrently
            work = []
            for nf, buf in gs:
                nbytes = c_size_t(0)
                with torch.cuda.device(dev):
                    _lib.check(self.lib.nfx_fft_work_bytes(self.precision, self.dim, _lib.int3(nf),
                                                           int(buf.shape[0]), byref(nbytes)), "nfx_fft_work_bytes")
                work.append(torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=dev))
            return gs, views, work

        self.groups, self.fw, self.fft_work = grid_set()
        self.groups2, self.fw2, self.fft_work2 = grid_set()

        # sort workspaces and batch problem tables
        self.opts = _lib.NfxOpts()
        self.opts.precision = self.precision
        self.opts.dim = self.dim
        self.opts.nf = _lib.int3((1, 1, 1))
        self.opts.nspread = self.kp.nspread
        self.opts.beta = self.kp.beta
        self.opts.kc = self.kp.c
        self.opts.prenorm = 1
        self.opts.tile = _lib.int3((0, 0, 0))
        self.opts.max_subproblem = 0
        self.ws = []
        probs_s = (_lib.NfxBatchProblem * self.P)()
        probs_i = (_lib.NfxBatchProblem * self.P)()
        for p in range(self.P):
            o = _lib.NfxOpts.from_buffer_copy(self.opts)
            o.nf = _lib.int3(self.nf[p])
            o.tile = _lib.int3(tiles[p] if tiles[p] is not None else (0, 0, 0))
            o.max_subproblem = int(maxsub[p] or 0)
            nbytes = ctypes.c_size_t(0)
            _lib.check(self.lib.nfx_sort_workspace_bytes(byref(o), self.M[p], byref(nbytes)), "workspace")
            ws = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=dev)
            self.ws.append(ws)
            for tab, src, dst in ((probs_s, self.c_in[p], self.fw[p]), (probs_i, self.fw2[p], self.c_out[p])):
                pb = tab[p]
                pb.M = self.M[p]
                cs = [t.data_ptr() for t in self.points[p]] + [None] * (3 - self.dim)
                pb.x, pb.y, pb.z = cs
                pb.nf = _lib.int3(self.nf[p])
                pb.tile = o.tile
                pb.max_subproblem = o.max_subproblem
                pb.interp_mode = int(imodes[p])
                pb.workspace = ws.data_ptr()
                pb.workspace_bytes = ws.numel()
                pb.src = src.data_ptr()
                pb.dst = dst.data_ptr()
        self._probs = probs_s  # keeps the struct array alive
        self._sort_opts = []
        for p in range(self.P):
            o = _lib.NfxOpts.from_buffer_copy(self.opts)
            o.nf = _lib.int3(self.nf[p])
            o.tile = probs_s[p].tile
            o.max_subproblem = probs_s[p].max_subproblem
            self._sort_opts.append(o)
        # independent per-problem sorts and per-class FFTs run on side streams
        # (fork / join), so the captured graph executes them concurrently; the
        # type-2 chain has its own stream and side streams for its FFTs
        self.n_side = min(8, self.P)
        self.side = [torch.cuda.Stream(device=self.device) for _ in range(self.n_side)]
        self.side2 = [torch.cuda.Stream(device=self.device) for _ in range(min(self.n_side, len(self.groups2)))]
        self.t2 = torch.cuda.Stream(device=self.device)
        self.info_s, self.table_s = self._upload(probs_s, spread=True)
        self.info_i, self.table_i = self._upload(probs_i, spread=False)
        # deconvolution tables
        facs = [[factors(self.nf[p][d], self.n_modes[p][d], self.kp, self.precision, dev) for d in range(self.dim)]
                for p in range(self.P)]
        self._facs = facs
        self.dtab_shuffle, self.dtotal_shuffle = self._deconv_table(pad=0, src=self.fw, dst=self.f_out)
        self.dtab_pad, self.dtotal_pad = self._deconv_table(pad=1, src=self.f_in, dst=self.fw2)
        self.graph = None
        self.use_graph = graph

    # -- set-up helpers -------------------------------------------------------
    def _upload(self, probs, spread: bool):
        info = _lib.NfxBatchInfo()
        _lib.check(self.lib.nfx_batch_info_get(byref(self.opts), int(spread), probs, self.P, byref(info)),
                   "nfx_batch_info_get")
        table = torch.empty(int(info.table_bytes), dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.nfx_batch_upload(byref(self.opts), int(spread), probs, self.P, ptr(table),
                                                 int(info.table_bytes), c_void_p(stream_of(self.device))),
                       "nfx_batch_upload")
        return info, table

    def _deconv_table(self, pad: int, src, dst):
        P = self.P
        nf = (c_int * (3 * P))()
        nm = (c_int * (3 * P))()
        fac = (c_void_p * (3 * P))()
        srcs = (c_void_p * P)()
        dsts = (c_void_p * P)()
        for p in range(P):
            for d in range(3):
                nf[3 * p + d] = self.nf[p][d] if d < self.dim else 1
                nm[3 * p + d] = self.n_modes[p][d] if d < self.dim else 1
                fac[3 * p + d] = self._facs[p][d].data_ptr() if d < self.dim else None
            srcs[p] = src[p].data_ptr()
            dsts[p] = dst[p].data_ptr()
        nbytes = int(self.lib.nfx_batch_deconv_table_bytes(self.precision, P))
        table = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        total = c_int64(0)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.nfx_batch_deconv_upload(self.precision, self.dim, pad, nf, nm, fac, srcs, dsts, P,
                                                        ptr(table), nbytes, byref(total),
                                                        c_void_p(stream_of(self.device))), "nfx_batch_deconv_upload")
        return table, int(total.value)

    # -- execution ------------------------------------------------------------
    @staticmethod
    def _fork(main, side, work):
        """Run work() on the `side` streams after `main`, then join them into `main`."""
        start = torch.cuda.Event()
        start.record(main)
        for sd in side:
            sd.wait_event(start)
        work()
        for sd in side:
            done = torch.cuda.Event()
            done.record(sd)
            main.wait_event(done)

    def _sorts(self):
        lib = self.lib
        for p in range(self.P):
            sd = self.side[p % self.n_side]
            cs = [t.data_ptr() for t in self.points[p]] + [None] * (3 - self.dim)
            _lib.check(lib.nfx_sort_points(byref(self._sort_opts[p]), c_void_p(cs[0]), c_void_p(cs[1]),
                                           c_void_p(cs[2]), self.M[p], ptr(self.ws[p]), self.ws[p].numel(),
                                           c_void_p(sd.cuda_stream)), "nfx_sort_points")

    def _ffts(self, sign, groups, works, side):
        lib = self.lib
        for i, (nf, buf) in enumerate(groups):
            sd = side[i % len(side)]
            work = works[i]
            _lib.check(lib.nfx_fft_ws(self.precision, self.dim, _lib.int3(nf), int(buf.shape[0]), ptr(buf), sign,
                                      ptr(work), work.numel(), c_void_p(sd.cuda_stream)), "nfx_fft_ws")

    def _enqueue(self):
        lib = self.lib
        main = torch.cuda.current_stream(self.device)
        st = c_void_p(main.cuda_stream)
        t2 = self.t2
        st2 = c_void_p(t2.cuda_stream)
        start = torch.cuda.Event()
        start.record(main)
        # sorts on the side streams, while the type-1 grids are zeroed on main
        for sd in self.side:
            sd.wait_event(start)
        self._sorts()
        for _, buf in self.groups:
            buf.zero_()
        sorted_ev = []
        for sd in self.side:
            ev = torch.cuda.Event()
            ev.record(sd)
            sorted_ev.append(ev)
            main.wait_event(ev)
        # type 2, on its own stream: deconvolve/pad and FFT run while the points
        # sort; the interpolation waits for the sorts
        t2.wait_event(start)
        _lib.check(lib.nfx_batch_deconv(self.precision, 1, ptr(self.dtab_pad), self.P, self.dtotal_pad, st2),
                   "nfx_batch_deconv(pad)")
        self._fork(t2, self.side2,
                   lambda: self._ffts(_fft_sign_type2(self.isign2), self.groups2, self.fft_work2, self.side2))
        for ev in sorted_ev:
            t2.wait_event(ev)
        _lib.check(lib.nfx_batch_launch(byref(self.opts), 0, ptr(self.table_i), self.P, byref(self.info_i), st2),
                   "nfx_batch_launch(interp)")
        # type 1 on the current stream
        _lib.check(lib.nfx_batch_launch(byref(self.opts), 1, ptr(self.table_s), self.P, byref(self.info_s), st),
                   "nfx_batch_launch(spread)")
        self._fork(main, self.side,
                   lambda: self._ffts(_fft_sign_type1(self.isign1), self.groups, self.fft_work, self.side))
        _lib.check(lib.nfx_batch_deconv(self.precision, 0, ptr(self.dtab_shuffle), self.P, self.dtotal_shuffle, st),
                   "nfx_batch_deconv(shuffle)")
        done2 = torch.cuda.Event()
        done2.record(t2)
        main.wait_event(done2)

    def run(self, c: Sequence[torch.Tensor] | None = None, f: Sequence[torch.Tensor] | None = None):
        """Type 1 of every problem's strengths and type 2 of its modes.

        Returns (f_out, c_out): lists of the plan's output tensors.
        """
        if c is not None:
            for dst, src in zip(self.c_in, c):
                dst.copy_(src, non_blocking=True)
        if f is not None:
            for dst, src in zip(self.f_in, f):
                dst.copy_(src, non_blocking=True)
        with torch.cuda.device(self.device):
            if not self.use_graph:
                self._enqueue()
            else:
                if self.graph is None:
                    self._enqueue()  # warm-up: creates cuFFT plans, sets kernel attributes
                    torch.cuda.current_stream(self.device).synchronize()
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        self._enqueue()
                    self.graph = g
                self.graph.replay()
        return self.f_out, self.c_out
