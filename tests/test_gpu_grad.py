"""GPU: hand-written adjoint kernels against the oracle and central finite differences.

Convention: torch's, G = dL/dRe + i dL/dIm (JAX's gradient is its conjugate;
the coordinate gradients are real and identical in both).
Finite differences run in complex128 with central steps on 32 random entries
(the reference's tests/test_adjoint.py checks the same quantities with
central FD at rtol 1e-6 in complex128).
"""

import numpy as np
import pytest
import torch

import nufftax_b200 as nb
from nufftax_b200.core import interp_2d, interp_3d, spread_1d, spread_2d, spread_3d, interp_1d
from oracle import nufft_oracle as O
from tests.conftest import cuda_device, rel_l2

pytestmark = pytest.mark.gpu


def dev():
    return cuda_device()


def T(a, grad=False):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(dev())
    return t.requires_grad_(grad)


def rand_c(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("dim,nf", [(1, (64,)), (2, (40, 36)), (3, (20, 18, 16))])
@pytest.mark.parametrize("n_trans", [1, 2])
def test_core_spread_grad_vs_oracle(dim, nf, n_trans):
    rng = np.random.default_rng(dim * 10 + n_trans)
    M = 400
    kp = nb.compute_kernel_params(1e-9)
    X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
    c = rand_c(rng, (n_trans, M))
    g = rand_c(rng, (n_trans,) + tuple(reversed(nf)))
    Xt = [T(x, True) for x in X]
    ct = T(c, True)
    fn = {1: spread_1d, 2: spread_2d, 3: spread_3d}[dim]
    out = fn(*Xt, ct, *nf, kp)
    out.backward(T(g))
    assert rel_l2(ct.grad.cpu().numpy(), O.interp(X, g, kp)) < 1e-12
    ref = O.spread_grad_coords(X, c, g, kp)
    for d in range(dim):
        assert rel_l2(Xt[d].grad.cpu().numpy(), ref[d]) < 1e-11


@pytest.mark.parametrize("dim,nf", [(1, (64,)), (2, (40, 36)), (3, (20, 18, 16))])
def test_core_interp_grad_vs_oracle(dim, nf):
    rng = np.random.default_rng(dim)
    M = 400
    kp = nb.compute_kernel_params(1e-9)
    X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
    fw = rand_c(rng, (2,) + tuple(reversed(nf)))
    g = rand_c(rng, (2, M))
    Xt = [T(x, True) for x in X]
    ft = T(fw, True)
    fn = {1: interp_1d, 2: interp_2d, 3: interp_3d}[dim]
    out = fn(*Xt, ft, *nf, kp)
    out.backward(T(g))
    assert rel_l2(ft.grad.cpu().numpy(), O.spread(X, g, nf, kp)) < 1e-12
    ref = O.interp_grad_coords(X, fw, g, kp)
    for d in range(dim):
        assert rel_l2(Xt[d].grad.cpu().numpy(), ref[d]) < 1e-11


def _fd_check(loss, params, rng, h, rtol, n_entries=32):
    """Central FD of a real scalar loss on random entries of each parameter."""
    loss(*params).backward()
    for p in params:
        if not p.requires_grad:
            continue
        g = p.grad.detach().cpu().numpy().ravel()
        base = p.detach().clone()
        idx = rng.choice(base.numel(), min(n_entries, base.numel()), replace=False)
        parts = [1.0] if not base.is_complex() else [1.0, 1j]
        for i in idx:
            for unit in parts:
                with torch.no_grad():
                    flat = p.view(-1)
                    flat[i] = base.view(-1)[i] + unit * h
                    lp = float(loss(*params))
                    flat[i] = base.view(-1)[i] - unit * h
                    lm = float(loss(*params))
                    flat[i] = base.view(-1)[i]
                fd = (lp - lm) / (2 * h)
                an = g[i].real if unit == 1.0 else g[i].imag
                assert abs(an - fd) <= rtol * max(1.0, abs(fd)), (i, unit, an, fd)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_type1_fd(dim):
    rng = np.random.default_rng(50 + dim)
    M = 60
    n_modes = {1: (16,), 2: (12, 10), 3: (8, 6, 6)}[dim]
    X = [T(rng.uniform(-np.pi, np.pi, M), True) for _ in range(dim)]
    c = T(rand_c(rng, M), True)
    target = T(rand_c(rng, tuple(reversed(n_modes))))
    fn = {1: nb.nufft1d1, 2: nb.nufft2d1, 3: nb.nufft3d1}[dim]
    nm = n_modes[0] if dim == 1 else n_modes

    def loss(*args):
        *xs, cc = args
        return (fn(*xs, cc, nm, eps=1e-10) - target).abs().pow(2).sum()

    _fd_check(loss, X + [c], rng, h=1e-5, rtol=1e-5)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_type2_fd(dim):
    rng = np.random.default_rng(60 + dim)
    M = 60
    shape = {1: (16,), 2: (10, 12), 3: (6, 6, 8)}[dim]
    X = [T(rng.uniform(-np.pi, np.pi, M), True) for _ in range(dim)]
    f = T(rand_c(rng, shape), True)
    target = T(rand_c(rng, M))
    fn = {1: nb.nufft1d2, 2: nb.nufft2d2, 3: nb.nufft3d2}[dim]

    def loss(*args):
        *xs, ff = args
        return (fn(*xs, ff, eps=1e-10) - target).abs().pow(2).sum()

    _fd_check(loss, X + [f], rng, h=1e-5, rtol=1e-5)


@pytest.mark.parametrize("dim", [1, 2])
def test_type3_fd(dim):
    rng = np.random.default_rng(70 + dim)
    M, K = 40, 30
    src = [T(rng.uniform(-np.pi, np.pi, M), True) for _ in range(dim)]
    tgt = [T(rng.uniform(-6, 6, K), True) for _ in range(dim)]
    c = T(rand_c(rng, M), True)
    target = T(rand_c(rng, K))
    nf = [O.type3_grid_size(np.pi, 6.0, 1e-10) for _ in range(dim)]
    fn = {1: nb.nufft1d3, 2: nb.nufft2d3}[dim]

    def loss(*args):
        xs, cc, ss = args[:dim], args[dim], args[dim + 1:]
        return (fn(*xs, cc, *ss, nf[0] if dim == 1 else nf, eps=1e-10) - target).abs().pow(2).sum()

    _fd_check(loss, src + [c] + tgt, rng, h=1e-5, rtol=2e-5, n_entries=8)


def test_type1_3d_grad_matches_spectral_reference_formula():
    """The ES-derivative adjoint equals the reference's spectral gradient
    (JVP k-weighted type 1 transposed into type 2, primitives.py:443-471) to eps."""
    rng = np.random.default_rng(80)
    M = 2000
    n_modes = (12, 10, 8)
    eps = 1e-10
    X = [rng.uniform(-np.pi, np.pi, M) for _ in range(3)]
    c = rand_c(rng, M)
    G = rand_c(rng, tuple(reversed(n_modes)))
    Xt = [T(x, True) for x in X]
    ct = T(c, True)
    nb.nufft3d1(*Xt, ct, n_modes, eps=eps).backward(T(G))
    # spectral form: dL/dx_d[j] = Re(conj(c_j) * type2(x, -i k_d G, isign=-1)_j)
    for d in range(3):
        shape = [1, 1, 1]
        shape[2 - d] = n_modes[d]
        k = O.mode_grid([n_modes[d]])[0].reshape(shape)
        t2 = O.nufft_type2(X, -1j * k * G, eps=eps, isign=-1)
        ref = np.real(np.conj(c) * t2)
        assert rel_l2(Xt[d].grad.cpu().numpy(), ref) < 1e-7
    assert rel_l2(ct.grad.cpu().numpy(), O.nufft_type2(X, G, eps=eps, isign=-1)) < 1e-9


def test_cg_least_squares_recovers_modes():
    """The linear-solve use of the reference (nufftax tests/test_linear_solve.py):
    conjugate gradients on the normal equations A^H A f = A^H c, with A the 2D
    type 2 (modes -> points, isign -1) and A^H the type 1 (isign +1), recovers
    the modes behind exact samples; the pair must be adjoint for CG to converge."""
    dev = cuda_device()
    rng = np.random.default_rng(17)
    M, n = 4000, (24, 20)
    x = torch.from_numpy(rng.uniform(-np.pi, np.pi, M)).to(dev)
    y = torch.from_numpy(rng.uniform(-np.pi, np.pi, M)).to(dev)
    f_true = torch.from_numpy(rng.standard_normal(n[::-1]) + 1j * rng.standard_normal(n[::-1])).to(dev)
    eps = 1e-12
    A = lambda f: nb.nufft2d2(x, y, f, eps=eps, isign=-1)  # noqa: E731
    AH = lambda c: nb.nufft2d1(x, y, c, n, eps=eps, isign=1)  # noqa: E731
    b = AH(A(f_true))
    f = torch.zeros_like(f_true)
    r = b.clone()
    p = r.clone()
    rr = torch.vdot(r.flatten(), r.flatten()).real
    for _ in range(60):
        Ap = AH(A(p))
        alpha = rr / torch.vdot(p.flatten(), Ap.flatten()).real
        f = f + alpha * p
        r = r - alpha * Ap
        rr_new = torch.vdot(r.flatten(), r.flatten()).real
        if float(rr_new.sqrt() / b.norm()) < 1e-11:
            break
        p = r + (rr_new / rr) * p
        rr = rr_new
    assert rel_l2(f.cpu().numpy(), f_true.cpu().numpy()) < 1e-8
