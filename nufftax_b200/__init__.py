"""nufftax_b200: B200-native (sm_100a) NUFFT hot path with nufftax's API.

Public transforms mirror nufftax (nufftax/__init__.py:54-98); every numerical
step runs in the CUDA library libnfx_b200.so (include/nfx.h).
"""

from .grid import (compute_grid_size, compute_type3_grid_size, compute_type3_grid_sizes_2d,
                   compute_type3_grid_sizes_3d, next_smooth_int)
from .kernel import KernelParams, compute_kernel_params, kernel_fourier_series
from .transforms import (nufft1d1, nufft1d1_jvp, nufft1d2, nufft1d2_jvp, nufft1d3, nufft1d3_jvp, nufft2d1,
                         nufft2d1_jvp, nufft2d2, nufft2d2_jvp, nufft2d3, nufft2d3_jvp, nufft3d1, nufft3d1_jvp,
                         nufft3d2, nufft3d2_jvp, nufft3d3, nufft3d3_jvp)
from ._plan import PointSort, clear_caches, sort_cache

__version__ = "0.1.0"

__all__ = [
    "nufft1d1", "nufft2d1", "nufft3d1",
    "nufft1d2", "nufft2d2", "nufft3d2",
    "nufft1d3", "nufft2d3", "nufft3d3",
    "nufft1d1_jvp", "nufft1d2_jvp", "nufft1d3_jvp",
    "nufft2d1_jvp", "nufft2d2_jvp", "nufft2d3_jvp",
    "nufft3d1_jvp", "nufft3d2_jvp", "nufft3d3_jvp",
    "compute_type3_grid_size", "compute_type3_grid_sizes_2d", "compute_type3_grid_sizes_3d",
    "compute_kernel_params", "compute_grid_size", "next_smooth_int", "kernel_fourier_series",
    "KernelParams", "PointSort", "clear_caches", "sort_cache",
]
