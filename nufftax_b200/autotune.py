"""Pick tile size, subproblem size and threads per point per (dim, upsampfac,
nspread, point density).

The tuner times sort + spread + interp on the caller's own points for a small
set of candidates (CUDA events, best of two runs each): tilings, and the
threads-per-point modes of the kernels (interpolation: one thread or one lane
group per point in 2D/3D; spread: one warp or the whole CTA per point in 3D).
The winner is cached under a key of dimension, upsampling factor, kernel width,
precision, a density bucket round(log2(M / prod(nf))) and a clustering flag
(largest bin holds more than 8x the mean).  The cache lives in memory and, when
NUFFTAX_B200_TUNE_CACHE names a file, in that JSON file too.
"""

from __future__ import annotations

import json
import math
import os
import threading
from typing import Sequence

import torch

from . import _lib
from ._plan import PointSort, complex_dtype
from .kernel import KernelParams

_TILINGS = {
    1: [((256,), 1024), ((512,), 1024), ((1024,), 2048)],
    2: [((16, 16), 512), ((32, 32), 1024), ((32, 32), 2048), ((64, 32), 2048), ((64, 64), 4096)],
    3: [((8, 8, 8), 1024), ((16, 16, 8), 2048), ((16, 16, 16), 4096)],
}
# (spread_mode, interp_mode) per dimension (NFX_PER_POINT_*)
_MODES = {
    1: [(_lib.NFX_PER_POINT_AUTO, _lib.NFX_PER_POINT_AUTO)],
    2: [(_lib.NFX_PER_POINT_WARP, _lib.NFX_PER_POINT_THREAD), (_lib.NFX_PER_POINT_WARP, _lib.NFX_PER_POINT_GROUP)],
    3: [(s, i) for s in (_lib.NFX_PER_POINT_WARP, _lib.NFX_PER_POINT_CTA)
        for i in (_lib.NFX_PER_POINT_THREAD, _lib.NFX_PER_POINT_GROUP)],
}

_lock = threading.Lock()
_cache: dict[str, tuple[tuple[int, ...], int, tuple[int, int]]] = {}
_loaded = False


def _cache_path():
    return os.environ.get("NUFFTAX_B200_TUNE_CACHE")


def _load():
    global _loaded
    if _loaded:
        return
    _loaded = True
    path = _cache_path()
    if path and os.path.exists(path):
        try:
            with open(path) as fh:
                for k, v in json.load(fh).items():
                    _cache[k] = (tuple(v[0]), int(v[1]), tuple(v[2]) if len(v) > 2 else (0, 0))
        except (OSError, ValueError):
            pass


def _save():
    path = _cache_path()
    if not path:
        return
    try:
        with open(path, "w") as fh:
            json.dump({k: [list(v[0]), v[1], list(v[2])] for k, v in _cache.items()}, fh)
    except OSError:
        pass


def density_key(coords: Sequence[torch.Tensor], nf: Sequence[int], kp: KernelParams) -> str:
    M = int(coords[0].shape[0])
    dens = round(math.log2(max(M, 1) / float(math.prod(nf))))
    ps = PointSort(coords, nf, kp, prenorm=True)
    _, _, bstart = ps.results()
    counts = (bstart[1:] - bstart[:-1]).float()
    clustered = bool(counts.max() > 8 * counts.mean().clamp(min=1e-9))
    prec = "f32" if coords[0].dtype == torch.float32 else "f64"
    return f"d{len(nf)}-uf{kp.upsampfac:g}-ns{kp.nspread}-{prec}-rho{dens}-{'clu' if clustered else 'uni'}"


def _time(coords, nf, kp, tile, maxsub, modes, c, fw) -> float:
    best = float("inf")
    for _ in range(2):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        ps = PointSort(coords, nf, kp, prenorm=True, tile=tile, max_subproblem=maxsub, modes=modes)
        ps.spread(c, out=fw)
        ps.interp(fw)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def tune(coords: Sequence[torch.Tensor], nf: Sequence[int], kp: KernelParams, timings: list | None = None
         ) -> tuple[tuple[int, ...], int, tuple[int, int]]:
    """(tile, max_subproblem, (spread_mode, interp_mode)) for these points on
    this grid (cached by class).  `timings`, when given, receives every
    candidate's (ms, tile, max_subproblem, modes)."""
    _load()
    key = density_key(coords, nf, kp)
    with _lock:
        if key in _cache:
            return _cache[key]
    dev = coords[0].device
    cdt = complex_dtype(0 if coords[0].dtype == torch.float32 else 1)
    M = int(coords[0].shape[0])
    c = torch.ones((1, M), dtype=cdt, device=dev)
    fw = torch.empty((1,) + tuple(reversed(nf)), dtype=cdt, device=dev)
    results = []
    for tile, maxsub in _TILINGS[len(nf)]:
        tile = tuple(min(t, n) for t, n in zip(tile, nf))
        for modes in _MODES[len(nf)]:
            try:
                results.append((_time(coords, nf, kp, tile, maxsub, modes, c, fw), tile, maxsub, modes))
            except (ValueError, NotImplementedError, RuntimeError):
                continue
    if timings is not None:
        timings.extend(results)
    _, tile, maxsub, modes = min(results)
    with _lock:
        _cache[key] = (tile, maxsub, modes)
        _save()
    return tile, maxsub, modes


def cached() -> dict:
    _load()
    return dict(_cache)
