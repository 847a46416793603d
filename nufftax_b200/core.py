"""Core spreading / interpolation (the seam nufftax routes to its GPU kernels).

Mirrors nufftax/core/spread.py: `spread_{1,2,3}d`, `interp_{1,2,3}d` (with the
custom VJPs of spread.py:766-1305, here torch.autograd.Functions whose backward
passes are the hand-written adjoint kernels) and the dispatch functions
`_spread_{1,2,3}d_dispatch` / `_interp_{1,2,3}d_dispatch` (spread.py:717-758)
that the transforms call.  Coordinates are taken as given (folded, not
pre-normalised), exactly like the reference core functions.

Gradient convention: torch's, G = dL/dRe + i dL/dIm.  The strength cotangent of
spread is interp(G) and the coordinate cotangent is
sum_t Re(conj(c_t) * sum_cells G_t dphi/dx) (spread.py:820-858); for interp the
grid cotangent is spread(G) and the coordinate cotangent
sum_t Re(conj(G_t) * sum_cells fw_t dphi/dx) (spread.py:911-944).
"""

from __future__ import annotations

from typing import Sequence

import torch

from ._plan import PointSort, precision_of, real_dtype, require_cuda, sort_cache
from .kernel import KernelParams


def _coords_for(coords: Sequence[torch.Tensor], dtype: torch.dtype) -> list[torch.Tensor]:
    out = []
    for c in coords:
        require_cuda(c, "coordinates")
        out.append(c.to(real_dtype(precision_of(dtype))).contiguous())
    return out


class _Spread(torch.autograd.Function):
    @staticmethod
    def forward(ctx, c, nf, kp, *coords):
        dim = len(coords)
        batched = c.ndim == 2
        c2 = (c if batched else c.unsqueeze(0)).contiguous()
        ps = sort_cache.get(list(coords), nf, kp, prenorm=False)
        fw = ps.spread(c2)
        ctx.ps = ps
        ctx.batched = batched
        ctx.save_for_backward(c2)
        return fw if batched else fw[0]

    @staticmethod
    def backward(ctx, g):
        (c2,) = ctx.saved_tensors
        ps: PointSort = ctx.ps
        need_c = ctx.needs_input_grad[0]
        need_x = list(ctx.needs_input_grad[3:])
        g2 = (g if ctx.batched else g.unsqueeze(0)).contiguous()
        dc, dxs = None, [None] * ps.dim
        if any(need_x):
            dc, dxs = ps.spread_grad(c2, g2, need_c, need_x)
        elif need_c:
            dc = ps.interp(g2)
        if dc is not None and not ctx.batched:
            dc = dc[0]
        return (dc, None, None, *dxs)


class _Interp(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fw, nf, kp, *coords):
        dim = len(coords)
        batched = fw.ndim == dim + 1
        fw2 = (fw if batched else fw.unsqueeze(0)).contiguous()
        ps = sort_cache.get(list(coords), nf, kp, prenorm=False)
        c = ps.interp(fw2)
        ctx.ps = ps
        ctx.batched = batched
        ctx.save_for_backward(fw2)
        return c if batched else c[0]

    @staticmethod
    def backward(ctx, g):
        (fw2,) = ctx.saved_tensors
        ps: PointSort = ctx.ps
        need_fw = ctx.needs_input_grad[0]
        need_x = list(ctx.needs_input_grad[3:])
        g2 = (g if ctx.batched else g.unsqueeze(0)).contiguous()
        dfw = ps.spread(g2) if need_fw else None
        dxs = ps.interp_grad(fw2, g2, need_x) if any(need_x) else [None] * ps.dim
        if dfw is not None and not ctx.batched:
            dfw = dfw[0]
        return (dfw, None, None, *dxs)


def _spread(coords, c, nf, kernel_params: KernelParams):
    coords = _coords_for(coords, c.dtype)
    require_cuda(c, "strengths")
    return _Spread.apply(c, tuple(int(n) for n in nf), kernel_params, *coords)


def _interp(coords, fw, kernel_params: KernelParams):
    dim = len(coords)
    coords = _coords_for(coords, fw.dtype)
    require_cuda(fw, "grid")
    nf = tuple(int(n) for n in reversed(fw.shape[-dim:]))
    return _Interp.apply(fw, nf, kernel_params, *coords)


# -- reference names: dispatch seam (nufftax/core/spread.py:717-758) ----------
def _spread_1d_dispatch(x, c, nf, kernel_params):
    return _spread([x], c, (nf,), kernel_params)


def _spread_2d_dispatch(x, y, c, nf1, nf2, kernel_params):
    return _spread([x, y], c, (nf1, nf2), kernel_params)


def _spread_3d_dispatch(x, y, z, c, nf1, nf2, nf3, kernel_params):
    return _spread([x, y, z], c, (nf1, nf2, nf3), kernel_params)


def _interp_1d_dispatch(x, fw, kernel_params):
    return _interp([x], fw, kernel_params)


def _interp_2d_dispatch(x, y, fw, kernel_params):
    return _interp([x, y], fw, kernel_params)


def _interp_3d_dispatch(x, y, z, fw, kernel_params):
    return _interp([x, y, z], fw, kernel_params)


# -- reference names: differentiable core functions (spread.py:766-1305) ------
def spread_1d(x, c, nf, kernel_params):
    """fw[k] = sum_j c[j] phi(k - fold(x[j]))  -> (n_trans?, nf)."""
    return _spread_1d_dispatch(x, c, nf, kernel_params)


def spread_2d(x, y, c, nf1, nf2, kernel_params):
    """2D spread -> (n_trans?, nf2, nf1), x fastest."""
    return _spread_2d_dispatch(x, y, c, nf1, nf2, kernel_params)


def spread_3d(x, y, z, c, nf1, nf2, nf3, kernel_params):
    """3D spread -> (n_trans?, nf3, nf2, nf1), x fastest."""
    return _spread_3d_dispatch(x, y, z, c, nf1, nf2, nf3, kernel_params)


def interp_1d(x, fw, nf, kernel_params):
    """c[j] = sum_k fw[k] phi(k - fold(x[j]))."""
    return _interp_1d_dispatch(x, fw, kernel_params)


def interp_2d(x, y, fw, nf1, nf2, kernel_params):
    return _interp_2d_dispatch(x, y, fw, kernel_params)


def interp_3d(x, y, z, fw, nf1, nf2, nf3, kernel_params):
    return _interp_3d_dispatch(x, y, z, fw, kernel_params)
