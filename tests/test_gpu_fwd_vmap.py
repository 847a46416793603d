"""GPU: forward-mode AD (torch.func.jvp, torch.autograd.forward_ad) and batching
(torch.func.vmap) of the transforms.

Forward mode follows the reference's JVP rules (nufftax/transforms/primitives.py:
type 1 and type 2 with k-weighted transforms, type 3 with s- and x-weighted
ones); each tangent is checked against central finite differences of the same
transform in complex128 (h = 1e-6, eps = 1e-12: truncation ~h^2 and rounding
~1e-16 / h, so agreement to 1e-7 relative).  vmap over strengths / modes must
equal a Python loop exactly up to float rounding (the batch becomes n_trans of
one call), and vmap over coordinates equals the loop too.
"""

import numpy as np
import pytest
import torch
import torch.autograd.forward_ad as fwAD

import nufftax_b200 as nb
from tests.conftest import cuda_device, rel_l2

pytestmark = pytest.mark.gpu

EPS = 1e-12
H = 1e-6


def dev():
    return cuda_device()


def rnd(rng, shape, cplx=False):
    a = rng.standard_normal(shape) + (1j * rng.standard_normal(shape) if cplx else 0)
    return torch.from_numpy(np.asarray(a)).to(dev())


def fd(fn, primals, tangents):
    plus = fn(*[p + H * t for p, t in zip(primals, tangents)])
    minus = fn(*[p - H * t for p, t in zip(primals, tangents)])
    return (plus - minus) / (2 * H)


T1 = {1: (nb.nufft1d1, 40), 2: (nb.nufft2d1, (24, 20)), 3: (nb.nufft3d1, (12, 10, 8))}
T2 = {1: nb.nufft1d2, 2: nb.nufft2d2, 3: nb.nufft3d2}


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("isign", [1, -1])
def test_jvp_type1_vs_finite_differences(dim, isign):
    rng = np.random.default_rng(40 + dim)
    M = 700
    fn0, nm = T1[dim]
    X = [rnd(rng, M) * 3.0 for _ in range(dim)]
    c = rnd(rng, (2, M), True)
    tX = [rnd(rng, M) for _ in range(dim)]
    tc = rnd(rng, (2, M), True)

    def fn(c, *X):
        return fn0(*X, c, nm, eps=EPS, isign=isign)

    out, tan = torch.func.jvp(fn, (c, *X), (tc, *tX))
    assert rel_l2(out.cpu().numpy(), fn(c, *X).cpu().numpy()) < 1e-14
    ref = fd(fn, (c, *X), (tc, *tX))
    assert rel_l2(tan.cpu().numpy(), ref.cpu().numpy()) < 1e-7
    # coordinates alone (c held fixed)
    _, tan_x = torch.func.jvp(lambda *X: fn(c, *X), tuple(X), tuple(tX))
    ref_x = fd(lambda *X: fn(c, *X), tuple(X), tuple(tX))
    assert rel_l2(tan_x.cpu().numpy(), ref_x.cpu().numpy()) < 1e-7


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_jvp_type2_vs_finite_differences(dim):
    rng = np.random.default_rng(50 + dim)
    M = 600
    nm = {1: (36,), 2: (20, 18), 3: (10, 12, 8)}[dim]
    X = [rnd(rng, M) * 3.0 for _ in range(dim)]
    f = rnd(rng, (2,) + tuple(reversed(nm)), True)
    tX = [rnd(rng, M) for _ in range(dim)]
    tf = rnd(rng, f.shape, True)

    def fn(f, *X):
        return T2[dim](*X, f, eps=EPS)

    _, tan = torch.func.jvp(fn, (f, *X), (tf, *tX))
    ref = fd(fn, (f, *X), (tf, *tX))
    assert rel_l2(tan.cpu().numpy(), ref.cpu().numpy()) < 1e-7


@pytest.mark.parametrize("dim", [1, 2])
def test_jvp_type3_vs_finite_differences(dim):
    rng = np.random.default_rng(60 + dim)
    M, K = 500, 400
    X = [torch.from_numpy(rng.uniform(-2.0, 2.0, M)).to(dev()) for _ in range(dim)]
    S = [torch.from_numpy(rng.uniform(-8.0, 8.0, K)).to(dev()) for _ in range(dim)]
    c = rnd(rng, M, True)
    # grid from half-widths with room for the finite-difference steps
    nf = [nb.compute_type3_grid_size(2.1, 8.1, eps=EPS) for _ in range(dim)]
    tX = [rnd(rng, M) for _ in range(dim)]
    tS = [rnd(rng, K) for _ in range(dim)]
    tc = rnd(rng, M, True)

    def fn(c, *P):
        if dim == 1:
            return nb.nufft1d3(P[0], c, P[1], nf[0], eps=EPS)
        return nb.nufft2d3(P[0], P[1], c, P[2], P[3], nf, eps=EPS)

    _, tan = torch.func.jvp(fn, (c, *X, *S), (tc, *tX, *tS))
    ref = fd(fn, (c, *X, *S), (tc, *tX, *tS))
    assert rel_l2(tan.cpu().numpy(), ref.cpu().numpy()) < 1e-7


def test_forward_ad_dual_tensors_and_jvp_alias():
    """torch.autograd.forward_ad through the *_jvp names (the same functions)."""
    rng = np.random.default_rng(7)
    M = 800
    x, y = rnd(rng, M) * 3.0, rnd(rng, M) * 3.0
    c = rnd(rng, M, True)
    tx, tc = rnd(rng, M), rnd(rng, M, True)
    assert nb.nufft2d1_jvp is nb.nufft2d1
    with fwAD.dual_level():
        f = nb.nufft2d1_jvp(fwAD.make_dual(x, tx), y, fwAD.make_dual(c, tc), (16, 14), eps=EPS)
        tan = fwAD.unpack_dual(f).tangent
    ref = fd(lambda c, x: nb.nufft2d1(x, y, c, (16, 14), eps=EPS), (c, x), (tc, tx))
    assert rel_l2(tan.cpu().numpy(), ref.cpu().numpy()) < 1e-7


@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_vmap_strengths_is_one_batched_call(prec):
    rng = np.random.default_rng(8)
    M, B = 3000, 5
    rdt = torch.float32 if prec == "c64" else torch.float64
    cdt = torch.complex64 if prec == "c64" else torch.complex128
    x, y = (rnd(rng, M) * 3.0).to(rdt), (rnd(rng, M) * 3.0).to(rdt)
    cs = rnd(rng, (M, B), True).to(cdt)  # batch on axis 1
    out = torch.func.vmap(lambda c: nb.nufft2d1(x, y, c, (32, 30), eps=1e-6), in_dims=1)(cs)
    loop = torch.stack([nb.nufft2d1(x, y, cs[:, b].contiguous(), (32, 30), eps=1e-6) for b in range(B)])
    assert out.shape == (B, 30, 32)
    assert rel_l2(out.cpu().numpy(), loop.cpu().numpy()) < (1e-6 if prec == "c64" else 1e-13)
    fs = rnd(rng, (B, 30, 32), True).to(cdt)
    c2 = torch.func.vmap(lambda f: nb.nufft2d2(x, y, f, eps=1e-6))(fs)
    loop2 = torch.stack([nb.nufft2d2(x, y, fs[b], eps=1e-6) for b in range(B)])
    assert rel_l2(c2.cpu().numpy(), loop2.cpu().numpy()) < (1e-6 if prec == "c64" else 1e-13)


def test_vmap_coordinates_and_type3():
    rng = np.random.default_rng(9)
    M, B = 1500, 3
    X = rnd(rng, (B, M)) * 3.0
    y = rnd(rng, M) * 3.0
    c = rnd(rng, M, True)
    out = torch.func.vmap(lambda x: nb.nufft2d1(x, y, c, (20, 20), eps=1e-9))(X)
    loop = torch.stack([nb.nufft2d1(X[b], y, c, (20, 20), eps=1e-9) for b in range(B)])
    assert rel_l2(out.cpu().numpy(), loop.cpu().numpy()) < 1e-13
    s = torch.from_numpy(rng.uniform(-10.0, 10.0, 900)).to(dev())
    cs = rnd(rng, (B, M), True)
    nf = nb.compute_type3_grid_size(y.cpu().numpy(), s.cpu().numpy(), eps=1e-9)
    o3 = torch.func.vmap(lambda cc: nb.nufft1d3(y, cc, s, nf, eps=1e-9))(cs)
    l3 = torch.stack([nb.nufft1d3(y, cs[b], s, nf, eps=1e-9) for b in range(B)])
    assert rel_l2(o3.cpu().numpy(), l3.cpu().numpy()) < 1e-13


def test_vmap_of_grad():
    """Per-example gradients: vmap over a batch of strengths of grad w.r.t. c."""
    rng = np.random.default_rng(10)
    M, B = 1000, 4
    x, y = rnd(rng, M) * 3.0, rnd(rng, M) * 3.0
    cs = rnd(rng, (B, M), True)
    tgt = rnd(rng, (12, 16), True)

    def loss(c):
        return (nb.nufft2d1(x, y, c, (16, 12), eps=1e-12) - tgt).abs().pow(2).sum()

    g = torch.func.vmap(torch.func.grad(loss))(cs)
    loop = []
    for b in range(B):
        cb = cs[b].clone().requires_grad_(True)
        loss(cb).backward()
        loop.append(cb.grad)
    assert rel_l2(g.cpu().numpy(), torch.stack(loop).cpu().numpy()) < 1e-12
