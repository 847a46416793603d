"""ES kernel parameters and Fourier coefficients (nufftax/core/kernel.py).

Host-side scalars: these run once per plan, in float64, and feed the CUDA kernels.
"""

from __future__ import annotations

import math
from typing import NamedTuple

import numpy as np


class KernelParams(NamedTuple):
    """Spreading-kernel parameters (nufftax/core/kernel.py:19-25)."""

    nspread: int
    beta: float
    c: float
    upsampfac: float


def compute_kernel_params(tol: float, upsampfac: float = 2.0, max_nspread: int = 16) -> KernelParams:
    """Kernel width and shape for a tolerance (nufftax/core/kernel.py:165-206).

    nspread = ceil(-log10 tol + 1), clamped to [2, max_nspread] and rounded up to
    even; beta = pi sqrt(ns^2 / sigma^2 (sigma - 1/2)^2 - 0.8) (2.3 ns if the root
    is not real); c = 4 / ns^2.
    """
    log_tol = -math.log10(max(tol, 1e-16))
    nspread = int(math.ceil(log_tol + 1))
    nspread = max(2, min(nspread, max_nspread))
    if nspread % 2 == 1:
        nspread += 1
    sigma = upsampfac
    inner = (nspread**2) / (sigma**2) * (sigma - 0.5) ** 2 - 0.8
    beta = math.pi * math.sqrt(inner) if inner > 0 else 2.3 * nspread
    return KernelParams(nspread=nspread, beta=beta, c=4.0 / (nspread**2), upsampfac=upsampfac)


def es_kernel(z: np.ndarray, beta: float, c: float) -> np.ndarray:
    """phi(z) = exp(beta (sqrt(1 - c z^2) - 1)), zero off the support (kernel.py:79-111)."""
    z = np.asarray(z)
    dt = z.dtype.type if np.issubdtype(z.dtype, np.floating) else np.float64
    z = z.astype(dt)
    arg = dt(1.0) - dt(c) * z * z
    val = np.exp(dt(beta) * (np.sqrt(np.maximum(arg, dt(0.0))) - dt(1.0)))
    return np.where(arg >= 0, val, dt(0.0))


def _trapezoid(nspread: int):
    j2 = nspread / 2.0
    n_quad = max(int(4 + 3.0 * j2), 20)
    z = np.linspace(-j2, j2, n_quad, dtype=np.float64)
    dz = z[1] - z[0]
    w = np.full(n_quad, dz)
    w[0] = w[-1] = dz / 2
    return z, w


def kernel_fourier_series(nf: int, nspread: int, beta: float, c: float) -> np.ndarray:
    """phihat[k] for k = 0..nf//2 by the trapezoid rule of kernel.py:209-260 (float64)."""
    z, w = _trapezoid(nspread)
    phi = es_kernel(z, beta, c)
    k = np.arange(nf // 2 + 1, dtype=np.float64)
    return (phi * w * np.cos(2.0 * np.pi * np.outer(k, z) / nf)).sum(axis=1)


def deconv_factors(nf: int, n_modes: int, kp: KernelParams) -> np.ndarray:
    """(-1)^k / phihat(|k|) for CMCL modes k = -n/2..(n-1)/2 (nufftax/core/deconvolve.py:27-56)."""
    ph = kernel_fourier_series(nf, kp.nspread, kp.beta, kp.c)
    k = np.arange(-(n_modes // 2), (n_modes - 1) // 2 + 1)
    return np.where(k % 2 == 0, 1.0, -1.0) / ph[np.abs(k)]
