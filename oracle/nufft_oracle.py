"""CPU oracle for the NUFFT hot path: a NumPy restatement of nufftax's pure-JAX path.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA path is
compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
legs of ``bench.py`` may import it; the product package ``nufftax_b200`` never does.

Every function cites the reference file:line it restates (paths are relative to
the nufftax project root, v0.6.0).  Arithmetic is dtype-faithful where the
reference's result depends on it bit-for-bit:

* coordinate pre-normalisation ``jnp.mod(x + pi, 2 pi) - pi`` and ``fold_rescale``
  run in the coordinate dtype with every Python constant rounded to that dtype
  first (JAX weak typing) and no fused multiply-add, so the integer cell/bin
  indices derived from them are exact;
* the ES weights are evaluated in the coordinate dtype;
* accumulations (segment_sum / gather-sum), the FFT and deconvolution run in
  float64 (the oracle is at least as accurate as the reference in float32).

Parity status: pinned to outputs of the reference's own source.  jax is not
installable here, so ``tests/golden/make_reference_golden.py`` runs nufftax's
pure-JAX modules unmodified on NumPy through ``tests/golden/jax_numpy_shim.py``
(a stand-in for the jax API subset they use, in the reference tests' x64
configuration) and stores seeded inputs with the reference's outputs in
``tests/golden/ref_*.npz``; ``tests/test_reference_golden.py`` holds this module
to them: the fold and pre-normalisation bit for bit, complex128 transforms, core
spread / interp and custom_vjp backward rules to 1e-12, complex64 within 2 eps
(the reference accumulates complex64 in float32).  The stand-in does not
reproduce XLA's fusion or scatter-add order, so the pin is to float rounding.
Also checked: the direct-DFT oracles of ``tests/conftest.py:154-198`` and
``tests/test_nufft3.py:26-72``, the known answers of ``tests/test_edge_cases.py``,
the adjoint identity of ``tests/test_spread.py:300-347`` and the kernel-parameter
table computed from ``nufftax/core/kernel.py:165-206``.
"""

from __future__ import annotations

import math
from typing import NamedTuple, Sequence

import numpy as np

# ---------------------------------------------------------------------------
# Kernel parameters and grid sizing
# ---------------------------------------------------------------------------


class KernelParams(NamedTuple):
    """nufftax/core/kernel.py:19-25."""

    nspread: int
    beta: float
    c: float
    upsampfac: float


def compute_kernel_params(tol: float, upsampfac: float = 2.0, max_nspread: int = 16) -> KernelParams:
    """nufftax/core/kernel.py:165-206 (ns from -log10 tol, forced even, FINUFFT beta)."""
    log_tol = -math.log10(max(tol, 1e-16))
    nspread = int(math.ceil(log_tol + 1))
    nspread = max(2, min(nspread, max_nspread))
    if nspread % 2 == 1:
        nspread += 1
    sigma = upsampfac
    inner = (nspread**2) / (sigma**2) * (sigma - 0.5) ** 2 - 0.8
    beta = math.pi * math.sqrt(inner) if inner > 0 else 2.3 * nspread
    return KernelParams(nspread, beta, 4.0 / (nspread**2), upsampfac)


def next_smooth_int(n: int) -> int:
    """nufftax/utils/grid.py:6-33: smallest 2,3,5-smooth integer >= n."""
    if n <= 1:
        return 1

    def smooth(v):
        for p in (2, 3, 5):
            while v % p == 0:
                v //= p
        return v == 1

    cand = n
    while not smooth(cand):
        cand += 1
    return cand


def compute_grid_size(n_modes: int, upsampfac: float, nspread: int) -> int:
    """nufftax/utils/grid.py:36-58."""
    return next_smooth_int(max(int(math.ceil(upsampfac * n_modes)), 2 * nspread))


def next_smooth_even(n: int) -> int:
    """nufftax/transforms/nufft3.py:35-47."""
    if n <= 1:
        return 2
    if n % 2 == 1:
        n += 1
    cand = next_smooth_int(n)
    while cand % 2 != 0:
        cand = next_smooth_int(cand + 1)
    return cand


def type3_grid_size(x_extent: float, s_extent: float, eps: float, upsampfac: float = 2.0) -> int:
    """nufftax/transforms/nufft3.py:50-106 (per-axis rule shared by 1D/2D/3D helpers)."""
    ns = compute_kernel_params(eps, upsampfac).nspread
    x_extent = max(float(x_extent), 1e-10)
    s_extent = max(float(s_extent), 1e-10)
    return next_smooth_even(int(np.ceil(2.0 * upsampfac * s_extent * x_extent / np.pi + ns)))


# ---------------------------------------------------------------------------
# ES kernel and its Fourier series
# ---------------------------------------------------------------------------


def es_kernel(z: np.ndarray, beta: float, c: float) -> np.ndarray:
    """nufftax/core/kernel.py:79-111, evaluated in z's dtype; arg = 1 - (c*z)*z."""
    dt = z.dtype.type
    arg = dt(1.0) - dt(c) * z * z
    res = np.exp(dt(beta) * (np.sqrt(np.maximum(arg, dt(0.0))) - dt(1.0)))
    return np.where(arg >= dt(0.0), res, dt(0.0)).astype(z.dtype)


def es_kernel_with_derivative(z: np.ndarray, beta: float, c: float):
    """nufftax/core/kernel.py:114-162 (dphi masked where arg <= 1e-14)."""
    dt = z.dtype.type
    arg = dt(1.0) - dt(c) * z * z
    sq = np.sqrt(np.maximum(arg, dt(1e-14)))
    phi = np.exp(dt(beta) * (sq - dt(1.0)))
    phi = np.where(arg >= dt(0.0), phi, dt(0.0))
    dphi = -dt(beta) * dt(c) * z / sq * phi
    dphi = np.where(arg > dt(1e-14), dphi, dt(0.0))
    return phi.astype(z.dtype), dphi.astype(z.dtype)


def _quad_nodes(nspread: int):
    """Shared by kernel.py:235-252 and nufft3.py:198-207: trapezoid on the support."""
    j2 = nspread / 2.0
    n_quad = max(int(4 + 3.0 * j2), 20)
    z = np.linspace(-j2, j2, n_quad, dtype=np.float64)
    dz = z[1] - z[0]
    w = np.full(n_quad, dz)
    w[0] = w[-1] = dz / 2
    return z, w


def kernel_fourier_series(nf: int, nspread: int, beta: float, c: float) -> np.ndarray:
    """nufftax/core/kernel.py:209-260: phihat[k], k = 0..nf//2, float64."""
    z, w = _quad_nodes(nspread)
    phi = es_kernel(z, beta, c)
    k = np.arange(nf // 2 + 1, dtype=np.float64)
    return (phi * w * np.cos(2.0 * np.pi * np.outer(k, z) / nf)).sum(axis=1)


def kernel_ft_at_point(k: np.ndarray, nspread: int, beta: float, c: float) -> np.ndarray:
    """nufftax/transforms/nufft3.py:176-213: phihat at arbitrary frequency, float64."""
    z, w = _quad_nodes(nspread)
    phi = es_kernel(z, beta, c)
    k = np.atleast_1d(np.asarray(k, dtype=np.float64))
    return (phi * w * np.cos(np.outer(k, z))).sum(axis=1)


# ---------------------------------------------------------------------------
# Coordinate folding (bit-exact in the coordinate dtype)
# ---------------------------------------------------------------------------


def premod(x: np.ndarray) -> np.ndarray:
    """jnp.mod(x + pi, 2*pi) - pi in x's dtype (nufftax/transforms/nufft1.py:71).

    jnp.mod on floats is lax.rem (C fmod, exact) plus a sign fix that adds the
    divisor when the truncated remainder is negative and non-zero.
    """
    dt = x.dtype.type
    pi = dt(np.pi)
    two_pi = dt(2.0 * np.pi)
    a = x + pi
    r = np.fmod(a, two_pi)
    r = np.where((r != dt(0)) & (r < dt(0)), r + two_pi, r).astype(x.dtype)
    return (r - pi).astype(x.dtype)


def fold_rescale(x: np.ndarray, nf: int) -> np.ndarray:
    """nufftax/core/spread.py:78-97: [-pi, pi) -> [0, nf], one rounding per op."""
    dt = x.dtype.type
    t = x * dt(1.0 / (2.0 * np.pi))
    t = t + dt(0.5)
    t = t - np.floor(t)
    return (t * dt(nf)).astype(x.dtype)


def cell_index(xs: np.ndarray, nspread: int) -> np.ndarray:
    """i0 = ceil(xs - ns/2) as int (nufftax/core/spread.py:214)."""
    dt = xs.dtype.type
    return np.ceil(xs - dt(nspread / 2.0)).astype(np.int64)


# ---------------------------------------------------------------------------
# Bin sort (no counterpart in the reference: defined here, mirrored on the GPU)
# ---------------------------------------------------------------------------


def bin_keys(coords: Sequence[np.ndarray], nf: Sequence[int], nspread: int, tile: Sequence[int],
             prenorm: bool):
    """(bin key, cell key) of every point.

    The point's left cell i0 = ceil(fold(x) - ns/2) is wrapped into [0, nf); its
    bin is i0 // tile per axis and its cell is i0 % tile per axis, both numbered
    x-fastest: bin = (bz * nby + by) * nbx + bx, cell = (lz * ty + ly) * tx + lx.
    """
    kb = np.zeros(coords[0].shape[0], dtype=np.int64)
    kc = np.zeros(coords[0].shape[0], dtype=np.int64)
    mb = mc = 1
    for d in range(len(coords)):
        x = premod(coords[d]) if prenorm else coords[d]
        i0 = cell_index(fold_rescale(x, nf[d]), nspread)
        i0w = np.mod(i0, nf[d])
        nb = -(-nf[d] // tile[d])
        kb += (i0w // tile[d]) * mb
        kc += (i0w % tile[d]) * mc
        mb *= nb
        mc *= tile[d]
    return kb.astype(np.int32), kc.astype(np.int32)


def bin_sort(kbin: np.ndarray, kcell: np.ndarray, nbins: int, ncell: int):
    """Stable sort by (bin, cell): (perm, bin_start), perm[k] = index of the k-th point."""
    fine = kbin.astype(np.int64) * ncell + kcell.astype(np.int64)
    perm = np.argsort(fine, kind="stable").astype(np.int32)
    counts = np.bincount(kbin, minlength=nbins)
    bin_start = np.zeros(nbins + 1, dtype=np.int64)
    np.cumsum(counts, out=bin_start[1:])
    return perm, bin_start.astype(np.int32)


# ---------------------------------------------------------------------------
# Weights, spread, interp
# ---------------------------------------------------------------------------


def _axis_weights(x: np.ndarray, nf: int, kp: KernelParams, derivative: bool = False):
    """nufftax/core/spread.py:187-277: wrapped indices (M, ns) and weights."""
    xs = fold_rescale(x, nf)
    i0 = cell_index(xs, kp.nspread)
    idx = i0[:, None] + np.arange(kp.nspread)[None, :]
    z = idx.astype(x.dtype) - xs[:, None]
    if derivative:
        w, dw = es_kernel_with_derivative(z, kp.beta, kp.c)
        scale = nf / (2.0 * np.pi)
        return np.mod(idx, nf), w.astype(np.float64), (-dw.astype(np.float64) * scale)
    return np.mod(idx, nf), es_kernel(z, kp.beta, kp.c).astype(np.float64)


def _flat_index_and_weights(coords, nf, kp):
    """Outer products over axes; flat index with x fastest (spread.py:466, 632-646)."""
    dim = len(coords)
    M = coords[0].shape[0]
    ns = kp.nspread
    idx = np.zeros((M,) + (1,) * dim, dtype=np.int64)
    w = np.ones((M,) + (1,) * dim, dtype=np.float64)
    stride = 1
    for d in range(dim):  # axis d of coordinates is array axis (dim-1-d) of the grid
        ii, ww = _axis_weights(coords[d], nf[d], kp)
        shape = [M] + [1] * dim
        shape[dim - d] = ns
        idx = idx + ii.reshape(shape) * stride
        w = w * ww.reshape(shape)
        stride *= nf[d]
    return idx.reshape(M, -1), w.reshape(M, -1)


# Points per chunk of the spread / interp sums: the (M, ns^d) index and weight
# tables of one chunk stay near 2^25 entries, so million-point inputs fit in
# memory.  Chunking changes only the order of the float64 sums.
_CHUNK_ENTRIES = 1 << 25


def _chunks(M: int, nspread: int, dim: int):
    step = max(1, _CHUNK_ENTRIES // (nspread ** dim))
    return [(s, min(s + step, M)) for s in range(0, M, step)]


def spread(coords: Sequence[np.ndarray], c: np.ndarray, nf: Sequence[int], kp: KernelParams) -> np.ndarray:
    """spread_{1,2,3}d_impl (nufftax/core/spread.py:285-339, 435-494, 596-658).

    coords: d arrays (M,) already in [-pi, pi) (fold handles any value).
    c: (M,) or (n_trans, M) complex.  Returns grid (n_trans?, nf_d..., nf_1), complex128.
    """
    c2 = c[None, :] if c.ndim == 1 else c
    ntot = int(np.prod(nf))
    out = np.zeros((c2.shape[0], ntot), dtype=np.complex128)
    for a, b in _chunks(coords[0].shape[0], kp.nspread, len(coords)):
        idx, w = _flat_index_and_weights([x[a:b] for x in coords], nf, kp)
        fi = idx.ravel()
        for t in range(c2.shape[0]):
            wc = (c2[t, a:b].astype(np.complex128)[:, None] * w).ravel()
            out[t] += np.bincount(fi, weights=wc.real, minlength=ntot) + 1j * np.bincount(
                fi, weights=wc.imag, minlength=ntot)
    out = out.reshape((c2.shape[0],) + tuple(reversed(nf)))
    return out[0] if c.ndim == 1 else out


def interp(coords: Sequence[np.ndarray], fw: np.ndarray, kp: KernelParams) -> np.ndarray:
    """interp_{1,2,3}d_impl (nufftax/core/spread.py:342-381, 497-540, 661-709)."""
    dim = len(coords)
    nf = tuple(reversed(fw.shape[-dim:]))
    batched = fw.ndim == dim + 1
    f2 = fw.reshape((-1, int(np.prod(nf)))).astype(np.complex128)
    M = coords[0].shape[0]
    out = np.empty((f2.shape[0], M), dtype=np.complex128)
    for a, b in _chunks(M, kp.nspread, dim):
        idx, w = _flat_index_and_weights([x[a:b] for x in coords], nf, kp)
        for t in range(f2.shape[0]):
            out[t, a:b] = (f2[t][idx] * w).sum(axis=1)
    return out if batched else out[0]


def _grad_parts(coords, nf, kp):
    per_axis = [_axis_weights(coords[d], nf[d], kp, derivative=True) for d in range(len(coords))]
    return per_axis


def _gather_with(per_axis, nf, which_deriv):
    """Flat indices and weights where axis `which_deriv` uses dphi (spread.py:997-1032)."""
    dim = len(per_axis)
    M = per_axis[0][0].shape[0]
    ns = per_axis[0][0].shape[1]
    idx = np.zeros((M,) + (1,) * dim, dtype=np.int64)
    w = np.ones((M,) + (1,) * dim, dtype=np.float64)
    stride = 1
    for d in range(dim):
        ii, ww, dw = per_axis[d]
        shape = [M] + [1] * dim
        shape[dim - d] = ns
        idx = idx + ii.reshape(shape) * stride
        w = w * (dw if d == which_deriv else ww).reshape(shape)
        stride *= nf[d]
    return idx.reshape(M, -1), w.reshape(M, -1)


def spread_grad_coords(coords, c, g, kp):
    """_spread_{1,2,3}d_grad_* (spread.py:820-858, 997-1032, 1168-1212).

    dx_d[j] = sum_t Re(conj(c[t,j]) * sum_cells g[t,cell] * dphi_d(cell)).
    """
    dim = len(coords)
    nf = tuple(reversed(g.shape[-dim:]))
    c2 = (c[None, :] if c.ndim == 1 else c).astype(np.complex128)
    g2 = g.reshape((-1, int(np.prod(nf)))).astype(np.complex128)
    per_axis = _grad_parts(coords, nf, kp)
    out = []
    for d in range(dim):
        idx, w = _gather_with(per_axis, nf, d)
        acc = np.zeros(coords[0].shape[0])
        for t in range(c2.shape[0]):
            acc += np.real(np.conj(c2[t]) * (g2[t][idx] * w).sum(axis=1))
        out.append(acc)
    return out


def interp_grad_coords(coords, fw, g, kp):
    """_interp_{1,2,3}d_grad_* (spread.py:911-944, 1080-1114, 1261-1305).

    dx_d[j] = sum_t Re(conj(g[t,j]) * sum_cells fw[t,cell] * dphi_d(cell)).
    """
    dim = len(coords)
    nf = tuple(reversed(fw.shape[-dim:]))
    f2 = fw.reshape((-1, int(np.prod(nf)))).astype(np.complex128)
    g2 = (g[None, :] if g.ndim == 1 else g).astype(np.complex128)
    per_axis = _grad_parts(coords, nf, kp)
    out = []
    for d in range(dim):
        idx, w = _gather_with(per_axis, nf, d)
        acc = np.zeros(coords[0].shape[0])
        for t in range(f2.shape[0]):
            acc += np.real(np.conj(g2[t]) * (f2[t][idx] * w).sum(axis=1))
        out.append(acc)
    return out


# ---------------------------------------------------------------------------
# Deconvolution / mode ordering
# ---------------------------------------------------------------------------


def deconv_factors_1d(phihat: np.ndarray, n_modes: int) -> np.ndarray:
    """nufftax/core/deconvolve.py:27-56 with modeord=0 (CMCL order, (-1)^k phase)."""
    kmin = -(n_modes // 2)
    kmax = (n_modes - 1) // 2
    k = np.arange(kmin, kmax + 1)
    fac = 1.0 / phihat[np.abs(k)]
    return np.where(k % 2 == 0, 1.0, -1.0) * fac


def extraction_indices_1d(nf: int, n_modes: int) -> np.ndarray:
    """nufftax/core/deconvolve.py:59-73 with modeord=0."""
    kmin = -(n_modes // 2)
    kmax = (n_modes - 1) // 2
    return np.concatenate([np.arange(nf + kmin, nf), np.arange(kmax + 1)])


def deconvolve_shuffle(fw_hat: np.ndarray, phihats, n_modes: Sequence[int]) -> np.ndarray:
    """deconvolve_shuffle_{1,2,3}d (nufftax/core/deconvolve.py:81-111, 174-224, 312-366).

    n_modes and phihats are ordered (axis 1 = x, axis 2 = y, axis 3 = z).
    """
    dim = len(n_modes)
    out = fw_hat
    for d in range(dim):
        ax = fw_hat.ndim - 1 - d
        nf = fw_hat.shape[ax]
        idx = extraction_indices_1d(nf, n_modes[d])
        fac = deconv_factors_1d(phihats[d], n_modes[d])
        shape = [1] * fw_hat.ndim
        shape[ax] = n_modes[d]
        out = np.take(out, idx, axis=ax) * fac.reshape(shape)
    return out


def deconvolve_pad(f: np.ndarray, phihats, nf: Sequence[int]) -> np.ndarray:
    """deconvolve_pad_{1,2,3}d (nufftax/core/deconvolve.py:114-166, 227-304, 369-468)."""
    dim = len(nf)
    out = f.astype(np.complex128)
    for d in range(dim):
        ax = f.ndim - 1 - d
        n = f.shape[ax]
        fac = deconv_factors_1d(phihats[d], n)
        shape = [1] * f.ndim
        shape[ax] = n
        out = out * fac.reshape(shape)
    full_shape = list(f.shape)
    for d in range(dim):
        full_shape[f.ndim - 1 - d] = nf[d]
    res = np.zeros(full_shape, dtype=np.complex128)
    index = [slice(None)] * f.ndim
    for d in range(dim):
        ax = f.ndim - 1 - d
        index[ax] = extraction_indices_1d(nf[d], f.shape[ax])
    res[np.ix_(*[np.arange(s) if isinstance(i, slice) else i for s, i in zip(res.shape, index)])] = out
    return res


# ---------------------------------------------------------------------------
# Transforms
# ---------------------------------------------------------------------------


def _fft(a, dim, isign, forward_for_negative=True):
    axes = tuple(range(a.ndim - dim, a.ndim))
    ntot = int(np.prod([a.shape[ax] for ax in axes]))
    if isign > 0:
        return np.fft.ifftn(a, axes=axes) * ntot
    return np.fft.fftn(a, axes=axes)


def nufft_type1(coords: Sequence[np.ndarray], c: np.ndarray, n_modes: Sequence[int], eps: float = 1e-6,
                isign: int = 1, upsampfac: float = 2.0) -> np.ndarray:
    """nufft{1,2,3}d1 (nufftax/transforms/nufft1.py:21-243).

    coords are (x[, y[, z]]); n_modes ordered (n1[, n2[, n3]]); output
    (n_trans?, n_d, ..., n_1) complex128.
    """
    dim = len(coords)
    kp = compute_kernel_params(eps, upsampfac)
    nf = [compute_grid_size(n, upsampfac, kp.nspread) for n in n_modes]
    ph = [kernel_fourier_series(n, kp.nspread, kp.beta, kp.c) for n in nf]
    xn = [premod(x) for x in coords]
    fw = spread(xn, c, nf, kp)
    fw_hat = _fft(fw, dim, isign)
    return deconvolve_shuffle(fw_hat, ph, n_modes)


def nufft_type2(coords: Sequence[np.ndarray], f: np.ndarray, eps: float = 1e-6, isign: int = -1,
                upsampfac: float = 2.0) -> np.ndarray:
    """nufft{1,2,3}d2 (nufftax/transforms/nufft2.py:21-227)."""
    dim = len(coords)
    kp = compute_kernel_params(eps, upsampfac)
    n_modes = [f.shape[f.ndim - 1 - d] for d in range(dim)]
    nf = [compute_grid_size(n, upsampfac, kp.nspread) for n in n_modes]
    ph = [kernel_fourier_series(n, kp.nspread, kp.beta, kp.c) for n in nf]
    fw_hat = deconvolve_pad(f, ph, nf)
    axes = tuple(range(fw_hat.ndim - dim, fw_hat.ndim))
    fw = np.fft.fftn(fw_hat, axes=axes) if isign < 0 else np.fft.ifftn(fw_hat, axes=axes) * int(np.prod(nf))
    xn = [premod(x) for x in coords]
    return interp(xn, fw, kp)


def nufft_type3(src: Sequence[np.ndarray], c: np.ndarray, tgt: Sequence[np.ndarray], n_modes: Sequence[int],
                eps: float = 1e-6, isign: int = 1, upsampfac: float = 2.0) -> np.ndarray:
    """nufft{1,2,3}d3 (nufftax/transforms/nufft3.py:216-515).

    Dtype-faithful like the fold: the centres, half-widths and scales
    (nufft3.py:258-268, 354-362) and the rescaled sources and targets
    (nufft3.py:271-272, 287-288, 365-366, 381-384) are computed in the
    coordinates' dtype in the reference's order, with Python constants rounded
    to that dtype first (JAX weak typing): C = (min + max) / 2,
    S = max((max - min) / 2, 1e-10), gamma = nf / ((2 upsampfac) S),
    x' = (x - C) / gamma, s' = (h gamma) (s - D) with h = 2 pi / nf.  The
    phases, phi-hat and the accumulations run in float64."""
    dim = len(src)
    kp = compute_kernel_params(eps, upsampfac)
    c2 = (c[None, :] if c.ndim == 1 else c).astype(np.complex128)
    dt = np.result_type(*[np.asarray(a).dtype for a in list(src) + list(tgt)])
    dt = np.dtype(np.float32) if dt == np.float32 else np.dtype(np.float64)
    t = dt.type
    src = [np.asarray(a, dtype=dt) for a in src]
    tgt = [np.asarray(a, dtype=dt) for a in tgt]
    C = [(a.min() + a.max()) / t(2.0) for a in src]
    D = [(a.min() + a.max()) / t(2.0) for a in tgt]
    S = [max((a.max() - a.min()) / t(2.0), t(1e-10)) for a in tgt]
    nf = list(n_modes)
    h = [2.0 * np.pi / n for n in nf]
    gam = [t(nf[d]) / (t(2.0 * upsampfac) * S[d]) for d in range(dim)]
    xn = [premod((src[d] - C[d]) / gam[d]) for d in range(dim)]
    phase_in = np.exp(1j * isign * sum(np.float64(D[d]) * src[d].astype(np.float64) for d in range(dim)))
    fw = spread(xn, c2 * phase_in[None, :], nf, kp)
    s_resc = [(t(h[d]) * gam[d]) * (tgt[d] - D[d]) for d in range(dim)]
    sn = [premod(a) for a in s_resc]
    f = nufft_type2(sn, fw, eps=eps, isign=isign, upsampfac=upsampfac)
    phi = np.ones(tgt[0].shape[0])
    for d in range(dim):
        phi = phi * kernel_ft_at_point(s_resc[d].astype(np.float64), kp.nspread, kp.beta, kp.c)
    ph = np.exp(1j * isign * sum((tgt[d].astype(np.float64) - np.float64(D[d])) * np.float64(C[d])
                                 for d in range(dim)))
    f = f * (ph / phi)[None, :]
    return f[0] if c.ndim == 1 else f


# ---------------------------------------------------------------------------
# Direct NUDFT oracles (float64)
# ---------------------------------------------------------------------------


def mode_grid(n_modes: Sequence[int]):
    """CMCL integer modes per axis: k = -n//2 .. (n-1)//2 (conftest.py:172)."""
    return [np.arange(-(n // 2), (n - 1) // 2 + 1) for n in n_modes]


def direct_type1(coords, c, n_modes, isign=1, flat_modes=None):
    """Direct sum f[k] = sum_j c_j exp(i isign k.x_j) (tests/conftest.py:154-175).

    flat_modes: optional (K, dim) integer modes to evaluate (subsample); else all.
    """
    dim = len(coords)
    c2 = (c[None, :] if c.ndim == 1 else c).astype(np.complex128)
    X = np.stack([np.asarray(a, dtype=np.float64) for a in coords], axis=1)
    full = flat_modes is None
    if full:
        flat_modes = flat_mode_list(n_modes)
    out = np.empty((c2.shape[0], flat_modes.shape[0]), dtype=np.complex128)
    for s in range(0, flat_modes.shape[0], 256):
        ph = np.exp(1j * isign * (flat_modes[s:s + 256].astype(np.float64) @ X.T))
        out[:, s:s + 256] = c2 @ ph.T
    if full:
        out = out.reshape((c2.shape[0],) + tuple(reversed(list(n_modes))))
    return out[0] if c.ndim == 1 else out


def flat_mode_list(n_modes: Sequence[int]) -> np.ndarray:
    """All CMCL modes as (K, dim) integer rows (k1, k2, k3), k1 fastest (array order)."""
    ks = mode_grid(list(reversed(list(n_modes))))
    mesh = np.meshgrid(*ks, indexing="ij")
    return np.stack([m.ravel() for m in reversed(mesh)], axis=1)


def direct_type2(coords, f_at_modes, flat_modes, isign=-1, rows=None):
    """Direct sum c_j = sum_k f_k exp(i isign k.x_j) (tests/conftest.py:178-198).

    f_at_modes: (n_trans?, K) values at flat_modes (K, dim); rows: optional point subset.
    """
    X = np.stack([np.asarray(a, dtype=np.float64) for a in coords], axis=1)
    if rows is not None:
        X = X[rows]
    f2 = f_at_modes[None, :] if f_at_modes.ndim == 1 else f_at_modes
    out = np.empty((f2.shape[0], X.shape[0]), dtype=np.complex128)
    for s in range(0, X.shape[0], 256):
        ph = np.exp(1j * isign * (X[s:s + 256] @ flat_modes.T.astype(np.float64)))
        out[:, s:s + 256] = f2 @ ph.T
    return out[0] if f_at_modes.ndim == 1 else out


def direct_type3(src, c, tgt, isign=1):
    """tests/test_nufft3.py:26-72: f_k = sum_j c_j exp(i isign s_k.x_j)."""
    X = np.stack([np.asarray(a, dtype=np.float64) for a in src], axis=1)
    S = np.stack([np.asarray(a, dtype=np.float64) for a in tgt], axis=1)
    c2 = (c[None, :] if c.ndim == 1 else c).astype(np.complex128)
    out = c2 @ np.exp(1j * isign * (X @ S.T))
    return out[0] if c.ndim == 1 else out


def direct_type1_product(coords, c, mode_axes, isign=1, chunk=1 << 18):
    """The direct sum of tests/conftest.py:154-175 at the product set of integer
    modes mode_axes = (k1 values, k2 values[, k3 values]), evaluated separably:
    exp(i isign k.x) = prod_d exp(i isign k_d x_d), so M points cost M * sum(len(k_d))
    exponentials and one matrix product per chunk of points,
    f[.., k2, k1] = sum_j (prod_{d>=2} E_d[j, k_d]) (c_j E_1[j, k1]).  Returns
    (len(k_d), ..., len(k_1)) complex128 (slowest axis first, as the transforms)."""
    dim = len(coords)
    M = coords[0].shape[0]
    ks = [np.asarray(k, dtype=np.float64) for k in mode_axes]
    sizes = [k.size for k in ks]
    out = np.zeros((int(np.prod(sizes[1:])), sizes[0]), dtype=np.complex128)
    c1 = np.asarray(c).astype(np.complex128)

    def expi(x, k):
        th = isign * np.outer(np.asarray(x, dtype=np.float64), k)
        return np.cos(th) + 1j * np.sin(th)

    for a in range(0, M, chunk):
        b = min(a + chunk, M)
        A = expi(coords[0][a:b], ks[0]) * c1[a:b, None]  # (m, n1)
        B = np.ones((b - a, 1), dtype=np.complex128)
        for d in range(1, dim):  # axis d becomes the new slowest axis of B
            B = (expi(coords[d][a:b], ks[d])[:, :, None] * B[:, None, :]).reshape(b - a, -1)
        out += B.T @ A
    return out.reshape(tuple(reversed(sizes)))


def direct_type2_points(points, f, isign=-1):
    """The direct sum of tests/conftest.py:178-198 at a few points (each of
    `points` holds the d coordinates of the same rows), over every CMCL mode of
    f (n_d, ..., n_1), contracted one axis at a time (x first)."""
    dim = len(points)
    n_modes = [f.shape[f.ndim - 1 - d] for d in range(dim)]
    ks = mode_grid(n_modes)
    X = [np.asarray(p, dtype=np.float64) for p in points]
    E = [np.exp(1j * isign * np.outer(X[d], ks[d])) for d in range(dim)]  # (J, n_d)
    G = np.tensordot(np.asarray(f, dtype=np.complex128), E[0].T, axes=([f.ndim - 1], [0]))  # (..., n2, J)
    for d in range(1, dim):
        # G: (n_{dim-1}.., n_d, J); contract n_d with E[d][j, :] row-wise
        G = np.einsum("...kj,jk->...j", G, E[d])
    return G


def modes_as_flat(f: np.ndarray, dim: int):
    """(n_trans?, n_d..n_1) CMCL array -> ((n_trans?, K) values, (K, dim) modes x-first)."""
    n_modes = [f.shape[f.ndim - 1 - d] for d in range(dim)]
    ks = mode_grid(list(reversed(n_modes)))  # array-axis order: slowest first
    mesh = np.meshgrid(*ks, indexing="ij")
    flat = np.stack([m.ravel() for m in reversed(mesh)], axis=1)  # columns (k1, k2, k3)
    lead = f.shape[:f.ndim - dim]
    return f.reshape(lead + (-1,)), flat


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
