"""CPU: the autograd layer of the transforms (reverse mode, forward mode, vmap).

The autograd Functions call the CUDA library only in their forward methods,
through five kernel-layer functions; here those are replaced by exact FP64
direct sums on CPU tensors (the NUDFT definitions of nufftax's tests,
tests/conftest.py:154-198), so the rules themselves are checked without a GPU:

  * jvp (torch.func.jvp and forward_ad dual tensors) against central finite
    differences, for every input of types 1, 2 and 3;
  * reverse mode against finite differences, and jacrev == jacfwd (the
    transpose rules agree with the JVP rules);
  * vmap over strengths / modes with shared points is ONE stacked call, and
    vmap over coordinates, vmap of grad and vmap of jvp equal Python loops.

The kernels themselves (the same functions on the GPU) are tested against the
oracle in the gpu-marked files.
"""

import numpy as np
import pytest
import torch
import torch.autograd.forward_ad as fwAD

from nufftax_b200 import transforms as T

H = 1e-6


def _modes(n_modes):
    return [torch.arange(-(n // 2), (n + 1) // 2, dtype=torch.float64) for n in n_modes]


def _flat_modes(n_modes):
    """(K, dim) integer modes, k1 fastest (the array order n_d..n_1)."""
    ks = _modes(n_modes)
    grids = torch.meshgrid(*reversed(ks), indexing="ij")
    return torch.stack([g.reshape(-1) for g in reversed(grids)], 1)


def _E(coords, n_modes, isign):
    K = _flat_modes(n_modes)
    X = torch.stack([c.to(torch.float64) for c in coords], 1)
    return torch.exp(1j * isign * (X @ K.T)), K


class Fakes:
    """Direct-sum stand-ins for the kernel layer (with call counts)."""

    def __init__(self):
        self.calls = {}

    def _n(self, name):
        self.calls[name] = self.calls.get(name, 0) + 1

    def t1(self, c2, n_modes, eps, isign, uf, coords):
        self._n("t1")
        E, _ = _E(coords, n_modes, isign)
        return (c2 @ E).reshape((c2.shape[0],) + tuple(reversed(n_modes)))

    def t2(self, f2, eps, isign, uf, coords):
        self._n("t2")
        n_modes = tuple(int(v) for v in reversed(f2.shape[1:]))
        E, _ = _E(coords, n_modes, isign)
        return f2.reshape(f2.shape[0], -1) @ E.T

    def t1_grad(self, c2, G, n_modes, eps, isign, uf_t, need_c, need_x, coords):
        self._n("t1_grad")
        E, K = _E(coords, n_modes, isign)
        Gf = G.reshape(G.shape[0], -1)
        dc = Gf @ E.conj().T if need_c else None
        dxs = [(c2.conj() * (Gf @ (E.conj() * (-1j * isign) * K[:, d][None, :]).T)).real.sum(0) if need_x[d]
               else None for d in range(len(coords))]
        return dc, dxs

    def t2_grad(self, f2, G, n_modes, eps, isign, uf, need_x, coords):
        self._n("t2_grad")
        E, K = _E(coords, n_modes, isign)
        ff = f2.reshape(f2.shape[0], -1)
        return [(G.conj() * (ff @ (E * (1j * isign) * K[:, d][None, :]).T)).real.sum(0) if need_x[d] else None
                for d in range(len(coords))]

    def t3(self, src, c2, tgt, nf, eps, isign, uf):
        self._n("t3")
        X = torch.stack(list(src), 1)
        S = torch.stack(list(tgt), 1)
        return c2 @ torch.exp(1j * isign * (X @ S.T))


@pytest.fixture
def fk(monkeypatch):
    f = Fakes()
    monkeypatch.setattr(T, "_type1_forward", f.t1)
    monkeypatch.setattr(T, "_type2_forward", f.t2)
    monkeypatch.setattr(T, "_type1_coord_grad", f.t1_grad)
    monkeypatch.setattr(T, "_type2_coord_grad", f.t2_grad)
    monkeypatch.setattr(T, "_type3_forward", f.t3)
    return f


NM = {1: (7,), 2: (6, 5), 3: (4, 5, 3)}


def t1(c, *X, isign=1):
    c2 = c if c.ndim == 2 else c.unsqueeze(0)
    f = T._Type1.apply(c2, NM[len(X)], 1e-9, isign, 2.0, 2.0, *X)
    return f if c.ndim == 2 else f[0]


def t2(f, *X, isign=-1):
    f2 = f if f.ndim == len(X) + 1 else f.unsqueeze(0)
    c = T._Type2.apply(f2, 1e-9, isign, 2.0, 2.0, *X)
    return c if f.ndim == len(X) + 1 else c[0]


def t3(c, *P, isign=1):
    dim = len(P) // 2
    c2 = c if c.ndim == 2 else c.unsqueeze(0)
    f = T._Type3.apply(c2, (32,) * dim, 1e-9, isign, 2.0, dim, *P)
    return f if c.ndim == 2 else f[0]


def rnd(rng, shape, cplx=False):
    a = rng.standard_normal(shape) + (1j * rng.standard_normal(shape) if cplx else 0)
    return torch.from_numpy(np.asarray(a))


def fd(fn, primals, tangents):
    plus = fn(*[p + H * t for p, t in zip(primals, tangents)])
    minus = fn(*[p - H * t for p, t in zip(primals, tangents)])
    return (plus - minus) / (2 * H)


def rel(a, b):
    return float((a - b).abs().pow(2).sum().sqrt() / b.abs().pow(2).sum().sqrt())


def inputs(rng, kind, dim, M=9, nt=None):
    X = [rnd(rng, M) for _ in range(dim)]
    if kind == 1:
        src = rnd(rng, (nt, M) if nt else M, True)
    elif kind == 2:
        src = rnd(rng, ((nt,) if nt else ()) + tuple(reversed(NM[dim])), True)
    else:
        src = rnd(rng, (nt, M) if nt else M, True)
        X = X + [rnd(rng, 8) for _ in range(dim)]
    return src, X


FN = {1: t1, 2: t2, 3: t3}


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_jvp_matches_finite_differences(fk, kind, dim):
    rng = np.random.default_rng(kind * 10 + dim)
    src, X = inputs(rng, kind, dim, nt=2)
    tangents = (rnd(rng, src.shape, True),) + tuple(rnd(rng, x.shape) for x in X)
    fn = FN[kind]
    out, tan = torch.func.jvp(fn, (src, *X), tangents)
    assert rel(out, fn(src, *X)) < 1e-14
    assert rel(tan, fd(fn, (src, *X), tangents)) < 1e-8
    # one input at a time (the others' tangents are absent, not zero)
    for i in range(1 + len(X)):
        def part(a, i=i):
            args = [src, *X]
            args[i] = a
            return fn(*args)
        p = ([src, *X])[i]
        _, ti = torch.func.jvp(part, (p,), (tangents[i],))
        assert rel(ti, fd(part, (p,), (tangents[i],))) < 1e-8


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_jvp_is_one_stacked_call(fk, kind):
    rng = np.random.default_rng(3)
    src, X = inputs(rng, kind, 2)
    tangents = (rnd(rng, src.shape, True),) + tuple(rnd(rng, x.shape) for x in X)
    fk.calls.clear()
    torch.func.jvp(FN[kind], (src, *X), tangents)
    name = {1: "t1", 2: "t2", 3: "t3"}[kind]
    assert fk.calls == {name: 2}  # the primal and ONE call for every tangent term


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("dim", [1, 2])
def test_reverse_mode_matches_finite_differences_and_jvp(fk, kind, dim):
    rng = np.random.default_rng(kind + 7 * dim)
    src, X = inputs(rng, kind, dim, nt=2)
    fn = FN[kind]
    W = rnd(rng, fn(src, *X).shape, True)

    def loss(*a):
        return (fn(*a) * W).real.sum() + fn(*a).abs().pow(2).sum()

    args = [a.clone().requires_grad_(True) for a in (src, *X)]
    grads = torch.autograd.grad(loss(*args), args)
    for i, g in enumerate(grads):
        t = rnd(rng, args[i].shape, args[i].is_complex())
        # directional derivative of the real loss along t: Re <g, t> in torch's convention
        dd = float((g.conj() * t).real.sum())
        ref = float(fd(loss, [a.detach() for a in args], [t if j == i else torch.zeros_like(a)
                                                          for j, a in enumerate(args)]))
        assert abs(dd - ref) <= 1e-7 * max(1.0, abs(ref))


def test_jacrev_equals_jacfwd(fk):
    rng = np.random.default_rng(11)
    X = [rnd(rng, 6) for _ in range(2)]
    c = rnd(rng, 6, True)
    for fn in (lambda x, y: t1(c, x, y).real, lambda x, y: t1(c, x, y).imag,
               lambda x, y: t2(rnd(np.random.default_rng(1), (5, 6), True), x, y).real):
        jr = torch.func.jacrev(fn, argnums=(0, 1))(*X)
        jf = torch.func.jacfwd(fn, argnums=(0, 1))(*X)
        for a, b in zip(jr, jf):
            assert rel(a, b) < 1e-12


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_vmap_over_strengths_is_one_call(fk, kind):
    rng = np.random.default_rng(5)
    B = 4
    src, X = inputs(rng, kind, 2, nt=B)  # the batch on axis 0
    fn = FN[kind]
    fk.calls.clear()
    out = torch.func.vmap(lambda s: fn(s, *X))(src)
    assert sum(fk.calls.values()) == 1
    loop = torch.stack([fn(src[b], *X) for b in range(B)])
    assert rel(out, loop) < 1e-14
    # batch on another axis of the input
    srcT = src.movedim(0, -1).contiguous()
    out2 = torch.func.vmap(lambda s: fn(s, *X), in_dims=-1)(srcT)
    assert rel(out2, loop) < 1e-14


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_vmap_over_coordinates_loops(fk, kind):
    rng = np.random.default_rng(6)
    B = 3
    src, X = inputs(rng, kind, 2)
    Xb = torch.stack([X[0] + 0.1 * b for b in range(B)])
    fn = FN[kind]
    out = torch.func.vmap(lambda x: fn(src, x, *X[1:]))(Xb)
    loop = torch.stack([fn(src, Xb[b], *X[1:]) for b in range(B)])
    assert rel(out, loop) < 1e-14


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_vmap_of_grad_per_example(fk, kind):
    rng = np.random.default_rng(7)
    B = 3
    src, X = inputs(rng, kind, 2, nt=B)
    fn = FN[kind]

    def loss(s, x):
        return fn(s, x, *X[1:]).abs().pow(2).sum()

    Xb = torch.stack([X[0] * (1 + 0.05 * b) for b in range(B)])
    gs, gx = torch.func.vmap(torch.func.grad(loss, argnums=(0, 1)))(src, Xb)
    for b in range(B):
        s = src[b].clone().requires_grad_(True)
        x = Xb[b].clone().requires_grad_(True)
        rs, rx = torch.autograd.grad(loss(s, x), (s, x))
        assert rel(gs[b], rs) < 1e-13 and rel(gx[b], rx) < 1e-13


def test_vmap_of_jvp_and_forward_ad(fk):
    rng = np.random.default_rng(8)
    c, X = inputs(rng, 1, 2)
    tb = rnd(rng, (3, 9), True)
    tans = torch.func.vmap(lambda t: torch.func.jvp(lambda cc: t1(cc, *X), (c,), (t,))[1])(tb)
    for b in range(3):
        assert rel(tans[b], t1(tb[b], *X)) < 1e-13  # linear in c
    tx = rnd(rng, 9)
    with fwAD.dual_level():
        f = t1(c, fwAD.make_dual(X[0], tx), X[1])
        tan = fwAD.unpack_dual(f).tangent
    assert rel(tan, fd(lambda x: t1(c, x, X[1]), (X[0],), (tx,))) < 1e-8


def test_second_derivative_in_strengths_only(fk):
    """Hessian-vector products in c go through the transpose rules (a type 2,
    then a type 1); second derivatives in the coordinates are refused."""
    rng = np.random.default_rng(9)
    c, X = inputs(rng, 1, 2)

    def loss(cr):
        return t1(cr.to(torch.complex128), *X).abs().pow(2).sum()

    cr = c.real.clone()
    hess = torch.func.hessian(loss)(cr)
    assert torch.allclose(hess, hess.T, atol=1e-10)
    xs = X[0].clone().requires_grad_(True)
    g, = torch.autograd.grad(t1(c, xs, X[1]).abs().pow(2).sum(), xs, create_graph=True)
    with pytest.raises(RuntimeError, match="second derivatives"):
        torch.autograd.grad(g.sum(), xs)
