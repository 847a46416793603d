"""Public NUFFT transforms nufft{1,2,3}d{1,2,3} (nufftax/transforms/autodiff.py:38-148).

Signatures, defaults, batching (leading n_trans axis), output layouts and the
`upsampfac` (forward, backward) tuple follow nufftax.  Inputs may be CUDA
tensors (results stay on the device), CPU tensors or numpy arrays (copied to the
current CUDA device and back).  Every numerical step runs in libnfx_b200:

  type 1 (nufftax/transforms/nufft1.py:21-243): bin sort -> spread -> cuFFT ->
         deconvolve + CMCL reorder + crop;
  type 2 (nufftax/transforms/nufft2.py:21-227): deconvolve + zero-pad -> cuFFT ->
         bin sort -> interp;
  type 3 (nufftax/transforms/nufft3.py:216-515): on-device centring/scaling and
         pre-phase -> spread -> inner type 2 -> phihat(s') and phase correction.

The three transforms are torch.autograd.Functions that take the place of the
JAX primitives of nufftax/transforms/primitives.py, with the same three rules:

  reverse mode (torch convention G = dL/dRe + i dL/dIm; the transpose rules):
    type 1: dc = type-2 adjoint pipeline of G; dx from the ES-derivative adjoint
            kernel on the same grid (one fused pass for dc, dx, dy, dz);
    type 2: df = type-1 adjoint pipeline of G; dx from the ES-derivative
            interpolation of the forward fine grid;
    type 3: dc, dx, ds through type-3 transforms of weighted cotangents
            (primitives.py:358-497);
  forward mode (torch.func.jvp, torch.autograd.forward_ad; the JVP rules
    _jvp_{1,2,3}d{1,2,3} of primitives.py:88-473): the tangent is the transform of
    dc (df) plus k-weighted transforms for the coordinate tangents, all of them
    stacked along n_trans into ONE call, so they share one sort and one launch
    of each kernel;
  batching (torch.func.vmap; the batcher of primitives.py:28-48): a batch of
    strengths / modes over shared coordinates becomes the n_trans axis of one
    call; batched coordinates run one call per batch element.

The `*_jvp` names are the same functions, as in nufftax (autodiff.py:150-161):
forward and reverse mode flow through the same Functions.
"""

from __future__ import annotations

from ctypes import byref, c_size_t, c_void_p
from typing import Sequence

import numpy as np
import torch
import torch.autograd.forward_ad as _fwad

from . import _lib
from ._plan import (_facs, complex_dtype, deconv_pad, deconv_shuffle, fft_inplace, make_opts, precision_of, ptr,
                    real_dtype, sort_cache, sort_launches, stream_of)
from .profiling import span
from .grid import compute_grid_size
from .kernel import compute_kernel_params


def _split_upsampfac(upsampfac) -> tuple[float, float]:
    """Scalar -> (uf, uf); (forward, backward) pair kept (autodiff.py:21-30)."""
    if isinstance(upsampfac, (tuple, list)):
        return float(upsampfac[0]), float(upsampfac[1])
    return float(upsampfac), float(upsampfac)


class _Boundary:
    """Moves host inputs to the device and results back to the caller's kind."""

    def __init__(self, *arrays):
        self.kind = "cuda"
        self.device = None
        for a in arrays:
            if isinstance(a, torch.Tensor) and a.is_cuda:
                self.device = a.device
                break
        if self.device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("nufftax_b200 needs a CUDA device (there is no CPU fallback)")
            self.device = torch.device("cuda", torch.cuda.current_device())
        for a in arrays:
            if isinstance(a, np.ndarray):
                self.kind = "numpy"
                break
            if isinstance(a, torch.Tensor) and not a.is_cuda:
                self.kind = "cpu"

    def to_dev(self, a, dtype=None) -> torch.Tensor:
        if isinstance(a, np.ndarray):
            a = torch.from_numpy(np.ascontiguousarray(a))
        elif not isinstance(a, torch.Tensor):
            a = torch.as_tensor(a)
        if a.device != self.device:
            a = a.to(self.device, non_blocking=True)
        if dtype is not None and a.dtype != dtype:
            a = a.to(dtype)
        return a

    def back(self, t: torch.Tensor):
        if self.kind == "cuda":
            return t
        t = t.detach().cpu() if self.kind == "numpy" else t.cpu()
        return t.numpy() if self.kind == "numpy" else t


def _precision_for(source) -> int:
    dt = source.dtype
    if isinstance(dt, np.dtype) or not isinstance(dt, torch.dtype):
        dt = torch.from_numpy(np.zeros(1, dtype=np.asarray(source).dtype)).dtype
    if dt in (torch.complex64, torch.float32, torch.float16, torch.bfloat16):
        return _lib.NFX_F32
    if dt in (torch.complex128, torch.float64):
        return _lib.NFX_F64
    raise TypeError(f"unsupported dtype {dt}")


def _fft_sign_type1(isign: int) -> int:
    # nufft1.py:81 -- isign > 0: ifft * nf (e^{+}); else fft (e^{-})
    return 1 if isign > 0 else -1


def _fft_sign_type2(isign: int) -> int:
    # nufft2.py:81 -- isign < 0: fft (e^{-}); else ifft * nf (e^{+})
    return -1 if isign < 0 else 1


_is_wrapped = torch._C._functorch.is_functorch_wrapped_tensor


def _tracked(*tensors) -> bool:
    """Whether the call must go through the autograd Function: an input needs a
    gradient, forward-mode AD is active, or a torch.func transform (vmap, jvp,
    grad) wraps an input.  Otherwise the forward runs directly, without
    autograd's bookkeeping."""
    if _fwad._current_level >= 0:
        return True
    grad = torch.is_grad_enabled()
    for t in tensors:
        if (grad and t.requires_grad) or _is_wrapped(t):
            return True
    return False


def _modes_axis(n: int, d: int, dim: int, device, dtype) -> torch.Tensor:
    """CMCL integer modes of axis d (k = -n/2 .. (n-1)/2) shaped to broadcast
    against a (n_trans, n_dim, ..., n_1) array."""
    k = torch.arange(-(n // 2), (n + 1) // 2, device=device, dtype=dtype)
    shape = [1] * (dim + 1)
    shape[dim - d] = n
    return k.reshape(shape)


def _bdim_front(t, bdim, B):
    """Batch axis moved to the front (an unbatched input is expanded)."""
    if bdim is None:
        return t.unsqueeze(0).expand((B,) + tuple(t.shape))
    return t.movedim(bdim, 0)


# ---------------------------------------------------------------------------
# Kernel layer: library calls on plain device tensors.  Only the forward
# methods of the autograd Functions below call these; their backward, jvp and
# vmap rules use Function.apply and torch operations only, so that torch.func
# transforms can unwrap the inputs level by level.
# ---------------------------------------------------------------------------
def _type1_forward(c2, n_modes, eps, isign, uf, coords):
    dim = len(coords)
    kp = compute_kernel_params(eps, uf)
    nf = tuple(compute_grid_size(n, uf, kp.nspread) for n in n_modes)
    ps = sort_cache.get(list(coords), nf, kp, prenorm=True)
    fw = ps.spread(c2)
    fft_inplace(fw, dim, _fft_sign_type1(isign))
    return deconv_shuffle(fw, n_modes, kp)


def _type1_coord_grad(c2, G, n_modes, eps, isign, uf_t, need_c, need_x, coords):
    """(dc or None, [dx_d or None]) of f = type 1 (c2 at coords) for the mode
    cotangent G: G deconvolved, zero-padded and transformed back onto the fine
    grid, then one fused ES-derivative pass over the points."""
    dim = len(coords)
    kp = compute_kernel_params(eps, uf_t)
    nf = tuple(compute_grid_size(n, uf_t, kp.nspread) for n in n_modes)
    H = deconv_pad(G.contiguous(), nf, kp)
    fft_inplace(H, dim, -_fft_sign_type1(isign))
    ps = sort_cache.get(list(coords), nf, kp, prenorm=True)
    return ps.spread_grad(c2.contiguous(), H, need_c, need_x)


def _type2_grid(f2, n_modes, eps, isign, uf, dim):
    kp = compute_kernel_params(eps, uf)
    nf = tuple(compute_grid_size(n, uf, kp.nspread) for n in n_modes)
    fw = deconv_pad(f2, nf, kp)
    fft_inplace(fw, dim, _fft_sign_type2(isign))
    return fw, nf, kp


def _type2_forward(f2, eps, isign, uf, coords):
    dim = len(coords)
    n_modes = tuple(int(v) for v in reversed(f2.shape[1:]))
    fw, nf, kp = _type2_grid(f2, n_modes, eps, isign, uf, dim)
    return sort_cache.get(list(coords), nf, kp, prenorm=True).interp(fw)


def _type2_coord_grad(f2, G, n_modes, eps, isign, uf, need_x, coords):
    """[dx_d or None] of c = type 2 (f2 at coords) for the point cotangent G:
    the forward fine grid again (deconvolve + FFT), then the ES-derivative
    interpolation on it."""
    dim = len(coords)
    fw, nf, kp = _type2_grid(f2.contiguous(), n_modes, eps, isign, uf, dim)
    return sort_cache.get(list(coords), nf, kp, prenorm=True).interp_grad(fw, G.contiguous(), need_x)


def _split_stack(F, nt, first):
    """Rows [0, nt) of a stacked call when `first` is set, and the offset of the next block."""
    return (F[:nt], nt) if first else (None, 0)


def _add(a, b):
    return b if a is None else a + b


# ---------------------------------------------------------------------------
# Type 1
# ---------------------------------------------------------------------------
class _Type1(torch.autograd.Function):
    """f = type 1 (c2 at coords), c2: (n_trans, M) -> (n_trans, N_d..N_1)."""

    @staticmethod
    def forward(c2, n_modes, eps, isign, uf, uf_t, *coords):
        return _type1_forward(c2, n_modes, eps, isign, uf, coords)

    @staticmethod
    def setup_context(ctx, inputs, output):
        c2, n_modes, eps, isign, uf, uf_t, *coords = inputs
        ctx.meta = (n_modes, eps, isign, uf, uf_t)
        ctx.save_for_backward(c2, *coords)
        ctx.save_for_forward(c2, *coords)

    @staticmethod
    def backward(ctx, G):
        c2, *coords = ctx.saved_tensors
        n_modes, eps, isign, uf, uf_t = ctx.meta
        need_c = ctx.needs_input_grad[0]
        need_x = tuple(ctx.needs_input_grad[6:])
        if any(need_x):
            dc, *dxs = _Type1CoordGrad.apply(c2, G, n_modes, eps, isign, uf_t, need_c, need_x, *coords)
        else:
            # transpose rule (_transpose_{1,2,3}d1, primitives.py:104, 191, 285):
            # type 2 of G with the upsampling factors swapped, and the sign
            # conjugated for torch's cotangent convention
            dxs = [None] * len(coords)
            dc = _Type2.apply(G.contiguous(), eps, -isign, uf_t, uf, *coords) if need_c else None
        return (dc, None, None, None, None, None, *dxs)

    @staticmethod
    def jvp(ctx, dc, _n, _e, _i, _u, _ut, *dxs):
        # df = T1(dc) + sum_d (i isign k_d) T1(c dx_d)   (_jvp_{1,2,3}d1, primitives.py:88, 170, 260)
        c2, *coords = ctx.saved_tensors
        n_modes, eps, isign, uf, uf_t = ctx.meta
        dim = len(coords)
        nt = c2.shape[0]
        parts = ([dc] if dc is not None else []) + [c2 * dx.to(c2.dtype)[None, :] for dx in dxs if dx is not None]
        if not parts:
            return None
        F = _Type1.apply(torch.cat(parts, 0).contiguous(), n_modes, eps, isign, uf, uf_t, *coords)
        out, i = _split_stack(F, nt, dc is not None)
        for d, dx in enumerate(dxs):
            if dx is not None:
                k = _modes_axis(n_modes[d], d, dim, F.device, F.real.dtype)
                out = _add(out, (1j * isign) * k * F[i:i + nt])
                i += nt
        return out

    @staticmethod
    def vmap(info, in_dims, c2, n_modes, eps, isign, uf, uf_t, *coords):
        cdim, xdims = in_dims[0], in_dims[6:]
        B = info.batch_size
        cb = _bdim_front(c2, cdim, B)
        if all(d is None for d in xdims):
            # shared points: the batch becomes part of n_trans (one call)
            nt = cb.shape[1]
            f = _Type1.apply(cb.reshape((B * nt,) + tuple(cb.shape[2:])), n_modes, eps, isign, uf, uf_t, *coords)
            return f.reshape((B, nt) + tuple(f.shape[1:])), 0
        xb = [_bdim_front(x, d, B) for x, d in zip(coords, xdims)]
        outs = [_Type1.apply(cb[b], n_modes, eps, isign, uf, uf_t, *[x[b] for x in xb]) for b in range(B)]
        return torch.stack(outs, 0), 0


class _Type1CoordGrad(torch.autograd.Function):
    """(dc, dx_1, .., dx_d) of a type 1 for the mode cotangent G (the fused
    ES-derivative adjoint pass).  Not differentiable itself: second derivatives
    with respect to the coordinates are not provided."""

    @staticmethod
    def forward(c2, G, n_modes, eps, isign, uf_t, need_c, need_x, *coords):
        dc, dxs = _type1_coord_grad(c2, G, n_modes, eps, isign, uf_t, need_c, need_x, coords)
        return (dc, *dxs)

    @staticmethod
    def setup_context(ctx, inputs, output):
        pass

    @staticmethod
    def backward(ctx, *grads):
        raise NotImplementedError("second derivatives with respect to the coordinates are not implemented")

    @staticmethod
    def vmap(info, in_dims, c2, G, n_modes, eps, isign, uf_t, need_c, need_x, *coords):
        # the coordinate gradients sum over n_trans, so batch elements stay apart
        B = info.batch_size
        cb, Gb = _bdim_front(c2, in_dims[0], B), _bdim_front(G, in_dims[1], B)
        xb = [_bdim_front(x, d, B) for x, d in zip(coords, in_dims[8:])]
        outs = [_Type1CoordGrad.apply(cb[b], Gb[b], n_modes, eps, isign, uf_t, need_c, need_x,
                                      *[x[b] for x in xb]) for b in range(B)]
        res = tuple(None if outs[0][i] is None else torch.stack([o[i] for o in outs]) for i in range(len(outs[0])))
        return res, tuple(None if r is None else 0 for r in res)


def _type1(coords, c, n_modes: Sequence[int], eps, isign, upsampfac):
    bd = _Boundary(c, *coords)
    precision = _precision_for(c)
    cd = bd.to_dev(c, complex_dtype(precision))
    xs = [bd.to_dev(x, real_dtype(precision)).contiguous() for x in coords]
    M = xs[0].shape[0]
    batched = cd.ndim == 2
    c2 = (cd if batched else cd.unsqueeze(0)).contiguous()
    if c2.shape[-1] != M:
        raise ValueError("c must have M entries along its last axis")
    uf, uf_t = _split_upsampfac(upsampfac)
    args = (c2, tuple(int(n) for n in n_modes), float(eps), int(isign), uf, uf_t, *xs)
    f = _Type1.apply(*args) if _tracked(c2, *xs) else _Type1.forward(*args)
    return bd.back(f if batched else f[0])


def nufft1d1(x, c, n_modes: int, eps: float = 1e-6, isign: int = 1, upsampfac=2.0):
    """f[k] = sum_j c[j] exp(i isign k x[j]), k = -N/2..(N-1)/2 -> (n_trans?, N)."""
    return _type1([x], c, (int(n_modes),), eps, isign, upsampfac)


def nufft2d1(x, y, c, n_modes, eps: float = 1e-6, isign: int = 1, upsampfac=2.0):
    """2D type 1 -> (n_trans?, N2, N1)."""
    n = (int(n_modes), int(n_modes)) if np.isscalar(n_modes) else tuple(int(v) for v in n_modes)
    return _type1([x, y], c, n, eps, isign, upsampfac)


def nufft3d1(x, y, z, c, n_modes, eps: float = 1e-6, isign: int = 1, upsampfac=2.0):
    """3D type 1 -> (n_trans?, N3, N2, N1)."""
    n = (int(n_modes),) * 3 if np.isscalar(n_modes) else tuple(int(v) for v in n_modes)
    return _type1([x, y, z], c, n, eps, isign, upsampfac)


# ---------------------------------------------------------------------------
# Type 2
# ---------------------------------------------------------------------------
class _Type2(torch.autograd.Function):
    """c = type 2 (f2 at coords), f2: (n_trans, N_d..N_1) -> (n_trans, M)."""

    @staticmethod
    def forward(f2, eps, isign, uf, uf_t, *coords):
        return _type2_forward(f2, eps, isign, uf, coords)

    @staticmethod
    def setup_context(ctx, inputs, output):
        f2, eps, isign, uf, uf_t, *coords = inputs
        ctx.meta = (tuple(int(v) for v in reversed(f2.shape[1:])), eps, isign, uf, uf_t)
        ctx.save_for_backward(f2, *coords)
        ctx.save_for_forward(f2, *coords)

    @staticmethod
    def backward(ctx, G):
        f2, *coords = ctx.saved_tensors
        n_modes, eps, isign, uf, uf_t = ctx.meta
        need_x = tuple(ctx.needs_input_grad[5:])
        # transpose rule (_transpose_{1,2,3}d2, primitives.py:145, 235, 334):
        # type 1 of G with the upsampling factors swapped, and the sign
        # conjugated for torch's cotangent convention
        df = _Type1.apply(G.contiguous(), n_modes, eps, -isign, uf_t, uf, *coords) if ctx.needs_input_grad[0] \
            else None
        dxs = list(_Type2CoordGrad.apply(f2, G, n_modes, eps, isign, uf, need_x, *coords)) if any(need_x) \
            else [None] * len(coords)
        return (df, None, None, None, None, *dxs)

    @staticmethod
    def jvp(ctx, df, _e, _i, _u, _ut, *dxs):
        # dc = T2(df) + sum_d dx_d T2(i isign k_d f)   (_jvp_{1,2,3}d2, primitives.py:127, 212, 306)
        f2, *coords = ctx.saved_tensors
        n_modes, eps, isign, uf, uf_t = ctx.meta
        dim = len(coords)
        nt = f2.shape[0]
        parts = [df] if df is not None else []
        for d, dx in enumerate(dxs):
            if dx is not None:
                parts.append((1j * isign) * _modes_axis(n_modes[d], d, dim, f2.device, f2.real.dtype) * f2)
        if not parts:
            return None
        C = _Type2.apply(torch.cat(parts, 0).contiguous(), eps, isign, uf, uf_t, *coords)
        out, i = _split_stack(C, nt, df is not None)
        for dx in dxs:
            if dx is not None:
                out = _add(out, dx.to(C.dtype)[None, :] * C[i:i + nt])
                i += nt
        return out

    @staticmethod
    def vmap(info, in_dims, f2, eps, isign, uf, uf_t, *coords):
        fdim, xdims = in_dims[0], in_dims[5:]
        B = info.batch_size
        fb = _bdim_front(f2, fdim, B)
        if all(d is None for d in xdims):
            nt = fb.shape[1]
            c = _Type2.apply(fb.reshape((B * nt,) + tuple(fb.shape[2:])), eps, isign, uf, uf_t, *coords)
            return c.reshape((B, nt) + tuple(c.shape[1:])), 0
        xb = [_bdim_front(x, d, B) for x, d in zip(coords, xdims)]
        outs = [_Type2.apply(fb[b], eps, isign, uf, uf_t, *[x[b] for x in xb]) for b in range(B)]
        return torch.stack(outs, 0), 0


class _Type2CoordGrad(torch.autograd.Function):
    """(dx_1, .., dx_d) of a type 2 for the point cotangent G (ES-derivative
    interpolation of the forward fine grid).  Not differentiable itself."""

    @staticmethod
    def forward(f2, G, n_modes, eps, isign, uf, need_x, *coords):
        return tuple(_type2_coord_grad(f2, G, n_modes, eps, isign, uf, need_x, coords))

    @staticmethod
    def setup_context(ctx, inputs, output):
        pass

    @staticmethod
    def backward(ctx, *grads):
        raise NotImplementedError("second derivatives with respect to the coordinates are not implemented")

    @staticmethod
    def vmap(info, in_dims, f2, G, n_modes, eps, isign, uf, need_x, *coords):
        B = info.batch_size
        fb, Gb = _bdim_front(f2, in_dims[0], B), _bdim_front(G, in_dims[1], B)
        xb = [_bdim_front(x, d, B) for x, d in zip(coords, in_dims[7:])]
        outs = [_Type2CoordGrad.apply(fb[b], Gb[b], n_modes, eps, isign, uf, need_x, *[x[b] for x in xb])
                for b in range(B)]
        res = tuple(None if outs[0][i] is None else torch.stack([o[i] for o in outs]) for i in range(len(outs[0])))
        return res, tuple(None if r is None else 0 for r in res)


def _type2(coords, f, eps, isign, upsampfac):
    dim = len(coords)
    bd = _Boundary(f, *coords)
    precision = _precision_for(f)
    fd = bd.to_dev(f, complex_dtype(precision))
    xs = [bd.to_dev(x, real_dtype(precision)).contiguous() for x in coords]
    batched = fd.ndim == dim + 1
    f2 = (fd if batched else fd.unsqueeze(0)).contiguous()
    uf, uf_t = _split_upsampfac(upsampfac)
    args = (f2, float(eps), int(isign), uf, uf_t, *xs)
    c = _Type2.apply(*args) if _tracked(f2, *xs) else _Type2.forward(*args)
    return bd.back(c if batched else c[0])


def nufft1d2(x, f, eps: float = 1e-6, isign: int = -1, upsampfac=2.0):
    """c[j] = sum_k f[k] exp(i isign k x[j]) -> (n_trans?, M)."""
    return _type2([x], f, eps, isign, upsampfac)


def nufft2d2(x, y, f, eps: float = 1e-6, isign: int = -1, upsampfac=2.0):
    """2D type 2; f is (n_trans?, N2, N1)."""
    return _type2([x, y], f, eps, isign, upsampfac)


def nufft3d2(x, y, z, f, eps: float = 1e-6, isign: int = -1, upsampfac=2.0):
    """3D type 2; f is (n_trans?, N3, N2, N1)."""
    return _type2([x, y, z], f, eps, isign, upsampfac)


# ---------------------------------------------------------------------------
# Type 3
# ---------------------------------------------------------------------------
def _type3_forward(src: list[torch.Tensor], c2: torch.Tensor, tgt: list[torch.Tensor], nf: tuple[int, ...],
                   eps: float, isign: int, uf: float, ws_alloc=None) -> torch.Tensor:
    """One nfx_nufft3 call: the type-3 scalars on the device, the source sort
    with the rescaling and pre-phase fused in, spread, the inner type 2's
    deconvolution / zero-pad and FFT, the target sort with the phase / phihat
    factor fused in, interpolation (nufftax/transforms/nufft3.py:216-515).
    ws_alloc(nbytes), when given, supplies the workspace (a caller's reusable
    buffer) instead of a fresh allocation."""
    dim = len(src)
    dev = c2.device
    precision = precision_of(c2.dtype)
    M = src[0].shape[0]
    K = tgt[0].shape[0]
    nt = c2.shape[0]
    kp = compute_kernel_params(eps, uf)
    lib = _lib.load()
    if M == 0 or K == 0:
        return torch.zeros((nt, K), dtype=c2.dtype, device=dev)
    nf = tuple(int(n) for n in nf)
    nf_in = tuple(compute_grid_size(n, uf, kp.nspread) for n in nf)
    opts = make_opts(precision, nf, kp, prenorm=False)
    nbytes = c_size_t(0)
    _lib.check(lib.nfx_nufft3_workspace_bytes(byref(opts), _lib.int3c(nf_in), M, K, nt, byref(nbytes)),
               "nfx_nufft3_workspace_bytes")
    ws = (ws_alloc or (lambda n: torch.empty(n, dtype=torch.uint8, device=dev)))(max(int(nbytes.value), 1))
    facs = _facs(nf_in, nf, kp, precision, dev)
    out = torch.empty((nt, K), dtype=c2.dtype, device=dev)
    arr = c_void_p * 3

    def parr(ts):
        return arr(*([t.data_ptr() for t in ts] + [None] * (3 - len(ts))))

    src = [a.contiguous() for a in src]
    tgt = [a.contiguous() for a in tgt]
    c2 = c2.contiguous()
    # our kernels: min / max per array, the scalars, both sorts, spread, zero-pad, interp
    launches = lambda: (2 * dim + 1 + sort_launches(opts, M, type3=True) + 2  # noqa: E731 (evaluated only when recording)
                        + sort_launches(make_opts(precision, nf_in, kp, prenorm=True), K, type3=True) + 1)
    with torch.cuda.device(dev), span("nfx_nufft3", dev, launches):
        _lib.check(lib.nfx_nufft3(byref(opts), _lib.int3c(nf_in), float(uf), int(isign), parr(src), M, ptr(c2), nt,
                                  parr(tgt), K, ptr(facs[0]), ptr(facs[1]), ptr(facs[2]), ptr(out), ptr(ws),
                                  ws.numel(), c_void_p(stream_of(dev))), "nfx_nufft3")
    return out


class _Type3(torch.autograd.Function):
    """f = type 3 (c2 at sources -> targets), c2: (n_trans, M) -> (n_trans, K)."""

    @staticmethod
    def forward(c2, nf, eps, isign, uf, dim, *pts):
        return _type3_forward(list(pts[:dim]), c2, list(pts[dim:]), nf, eps, isign, uf)

    @staticmethod
    def setup_context(ctx, inputs, output):
        c2, nf, eps, isign, uf, dim, *pts = inputs
        ctx.meta = (nf, eps, isign, uf, dim)
        ctx.save_for_backward(c2, *pts)
        ctx.save_for_forward(c2, *pts)

    @staticmethod
    def backward(ctx, G):
        # _transpose_{1,2,3}d3 (primitives.py:376, 422, 473) and the coordinate
        # terms of the JVP rules, transposed: the conjugate transpose is a type 3 from the
        # targets to the sources with -isign; the coordinate terms are weighted
        # transforms.  Each direction is one stacked call.
        c2, *pts = ctx.saved_tensors
        nf, eps, isign, uf, dim = ctx.meta
        src, tgt = list(pts[:dim]), list(pts[dim:])
        nt = c2.shape[0]
        need_c = ctx.needs_input_grad[0]
        need_x = ctx.needs_input_grad[6:6 + dim]
        need_s = ctx.needs_input_grad[6 + dim:]
        G = G.contiguous()
        dc, gx, gs = None, [None] * dim, [None] * dim
        parts = ([G] if need_c else []) + [(-1j * isign) * tgt[d].to(G.dtype)[None, :] * G
                                           for d in range(dim) if need_x[d]]
        if parts:
            T = _Type3.apply(torch.cat(parts, 0).contiguous(), nf, eps, -isign, uf, dim, *tgt, *src)
            dc, i = _split_stack(T, nt, need_c)
            for d in range(dim):
                if need_x[d]:
                    gx[d] = (c2.conj() * T[i:i + nt]).real.sum(0)
                    i += nt
        parts = [src[d].to(c2.dtype)[None, :] * c2 for d in range(dim) if need_s[d]]
        if parts:
            F = _Type3.apply(torch.cat(parts, 0).contiguous(), nf, eps, isign, uf, dim, *src, *tgt)
            i = 0
            for d in range(dim):
                if need_s[d]:
                    gs[d] = (G.conj() * (1j * isign) * F[i:i + nt]).real.sum(0)
                    i += nt
        return (dc, None, None, None, None, None, *gx, *gs)

    @staticmethod
    def jvp(ctx, dc, _nf, _e, _i, _u, _d, *dpts):
        # df = T3(dc) + sum_d (i isign s_d) T3(c dx_d) + sum_d (i isign ds_d) T3(x_d c)
        # (_jvp_{1,2,3}d3, primitives.py:358, 398, 443), all strengths stacked into one call
        c2, *pts = ctx.saved_tensors
        nf, eps, isign, uf, dim = ctx.meta
        src, tgt = pts[:dim], pts[dim:]
        nt = c2.shape[0]
        dxs, dss = dpts[:dim], dpts[dim:]
        parts = [dc] if dc is not None else []
        parts += [c2 * dx.to(c2.dtype)[None, :] for dx in dxs if dx is not None]
        parts += [src[d].to(c2.dtype)[None, :] * c2 for d in range(dim) if dss[d] is not None]
        if not parts:
            return None
        F = _Type3.apply(torch.cat(parts, 0).contiguous(), nf, eps, isign, uf, dim, *pts)
        out, i = _split_stack(F, nt, dc is not None)
        for d, dx in enumerate(dxs):
            if dx is not None:
                out = _add(out, (1j * isign) * tgt[d].to(F.dtype)[None, :] * F[i:i + nt])
                i += nt
        for d, ds in enumerate(dss):
            if ds is not None:
                out = _add(out, (1j * isign) * ds.to(F.dtype)[None, :] * F[i:i + nt])
                i += nt
        return out

    @staticmethod
    def vmap(info, in_dims, c2, nf, eps, isign, uf, dim, *pts):
        cdim, pdims = in_dims[0], in_dims[6:]
        B = info.batch_size
        cb = _bdim_front(c2, cdim, B)
        if all(d is None for d in pdims):
            nt = cb.shape[1]
            f = _Type3.apply(cb.reshape((B * nt,) + tuple(cb.shape[2:])), nf, eps, isign, uf, dim, *pts)
            return f.reshape((B, nt) + tuple(f.shape[1:])), 0
        pb = [_bdim_front(p, d, B) for p, d in zip(pts, pdims)]
        outs = [_Type3.apply(cb[b], nf, eps, isign, uf, dim, *[p[b] for p in pb]) for b in range(B)]
        return torch.stack(outs, 0), 0


def _type3(src, c, tgt, n_modes, eps, isign, upsampfac):
    dim = len(src)
    bd = _Boundary(c, *src, *tgt)
    precision = _precision_for(c)
    cd = bd.to_dev(c, complex_dtype(precision))
    xs = [bd.to_dev(a, real_dtype(precision)).contiguous() for a in src]
    ss = [bd.to_dev(a, real_dtype(precision)).contiguous() for a in tgt]
    batched = cd.ndim == 2
    c2 = (cd if batched else cd.unsqueeze(0)).contiguous()
    nf = (int(n_modes),) if dim == 1 and np.isscalar(n_modes) else tuple(int(v) for v in n_modes)
    if len(nf) != dim:
        raise ValueError(f"n_modes must have {dim} entries")
    args = (c2, nf, float(eps), int(isign), float(upsampfac), dim, *xs, *ss)
    f = _Type3.apply(*args) if _tracked(c2, *xs, *ss) else _Type3.forward(*args)
    return bd.back(f if batched else f[0])


def nufft1d3(x, c, s, n_modes: int, eps: float = 1e-6, isign: int = 1, upsampfac: float = 2.0):
    """f[k] = sum_j c[j] exp(i isign s[k] x[j]); n_modes from compute_type3_grid_size."""
    return _type3([x], c, [s], n_modes, eps, isign, upsampfac)


def nufft2d3(x, y, c, s, t, n_modes, eps: float = 1e-6, isign: int = 1, upsampfac: float = 2.0):
    """2D type 3; n_modes = (nf1, nf2) from compute_type3_grid_sizes_2d."""
    return _type3([x, y], c, [s, t], n_modes, eps, isign, upsampfac)


def nufft3d3(x, y, z, c, s, t, u, n_modes, eps: float = 1e-6, isign: int = 1, upsampfac: float = 2.0):
    """3D type 3; n_modes = (nf1, nf2, nf3) from compute_type3_grid_sizes_3d."""
    return _type3([x, y, z], c, [s, t, u], n_modes, eps, isign, upsampfac)


# The *_jvp names of nufftax (autodiff.py:150-161): the same functions, whose
# autograd Functions carry the forward-mode (jvp) and batching (vmap) rules.
nufft1d1_jvp = nufft1d1
nufft1d2_jvp = nufft1d2
nufft2d1_jvp = nufft2d1
nufft2d2_jvp = nufft2d2
nufft3d1_jvp = nufft3d1
nufft3d2_jvp = nufft3d2
nufft1d3_jvp = nufft1d3
nufft2d3_jvp = nufft2d3
nufft3d3_jvp = nufft3d3
