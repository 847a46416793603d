"""Fine-grid sizing (nufftax/utils/grid.py:6-58, nufftax/transforms/nufft3.py:35-173)."""

from __future__ import annotations

import math

import numpy as np

from .kernel import compute_kernel_params


def next_smooth_int(n: int) -> int:
    """Smallest integer >= n whose only prime factors are 2, 3 and 5 (grid.py:6-33)."""
    if n <= 1:
        return 1
    cand = n
    while True:
        v = cand
        for p in (2, 3, 5):
            while v % p == 0:
                v //= p
        if v == 1:
            return cand
        cand += 1


def compute_grid_size(n_modes: int, upsampfac: float, nspread: int) -> int:
    """nf = smooth(max(ceil(upsampfac * n_modes), 2 * nspread)) (grid.py:36-58)."""
    return next_smooth_int(max(int(math.ceil(upsampfac * n_modes)), 2 * nspread))


def _next_smooth_even(n: int) -> int:
    """Next even 2,3,5-smooth integer >= n (nufft3.py:35-47)."""
    if n <= 1:
        return 2
    if n % 2 == 1:
        n += 1
    cand = next_smooth_int(n)
    while cand % 2 != 0:
        cand = next_smooth_int(cand + 1)
    return cand


def _extent(a) -> float:
    arr = np.asarray(a.detach().cpu() if hasattr(a, "detach") else a)
    if arr.ndim > 0:
        return float((np.max(arr) - np.min(arr)) / 2)
    return float(arr)


def _axis_size(x_extent: float, s_extent: float, nspread: int, upsampfac: float) -> int:
    x_extent = max(x_extent, 1e-10)
    s_extent = max(s_extent, 1e-10)
    return _next_smooth_even(int(np.ceil(2.0 * upsampfac * s_extent * x_extent / np.pi + nspread)))


def compute_type3_grid_size(x_or_x_extent, s_or_s_extent, eps: float = 1e-6, upsampfac: float = 2.0) -> int:
    """1D type-3 grid size from point arrays or half-widths (nufft3.py:50-106)."""
    ns = compute_kernel_params(eps, upsampfac).nspread
    return _axis_size(_extent(x_or_x_extent), _extent(s_or_s_extent), ns, upsampfac)


def compute_type3_grid_sizes_2d(x_extent, y_extent, s_extent, t_extent, eps: float = 1e-6,
                                upsampfac: float = 2.0) -> tuple[int, int]:
    """2D type-3 grid sizes from half-widths (nufft3.py:109-135)."""
    ns = compute_kernel_params(eps, upsampfac).nspread
    return (_axis_size(float(x_extent), float(s_extent), ns, upsampfac),
            _axis_size(float(y_extent), float(t_extent), ns, upsampfac))


def compute_type3_grid_sizes_3d(x_extent, y_extent, z_extent, s_extent, t_extent, u_extent, eps: float = 1e-6,
                                upsampfac: float = 2.0) -> tuple[int, int, int]:
    """3D type-3 grid sizes from half-widths (nufft3.py:138-173)."""
    ns = compute_kernel_params(eps, upsampfac).nspread
    return (_axis_size(float(x_extent), float(s_extent), ns, upsampfac),
            _axis_size(float(y_extent), float(t_extent), ns, upsampfac),
            _axis_size(float(z_extent), float(u_extent), ns, upsampfac))
