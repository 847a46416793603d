"""GPU: the CUDA path against golden vectors computed by the reference's own source.

tests/golden/ref_*.npz come from make_reference_golden.py (nufftax's pure-JAX
modules run unmodified on NumPy through jax_numpy_shim.py).  Bars, as in the
CPU pin of the oracle: relative l2 <= 2 eps for the transforms (5 eps for
complex64 at upsampfac 1.25, where the reference's float32 accumulation alone
is 3e-6 away from float64 arithmetic); bit-exact bin keys from the reference's
fold_rescale; 1e-12 for the complex128 core spread / interp and the
custom_vjp backward rules (spread.py:766-1305), whose formulas the autograd
Functions of nufftax_b200.core follow.
"""

import numpy as np
import pytest
import torch

import nufftax_b200 as nb
from nufftax_b200 import PointSort
from nufftax_b200.core import interp_2d, interp_3d, spread_2d, spread_3d
from tests.conftest import GOLDEN, cuda_device, rel_l2
from tests.test_reference_golden import _cases, _parse, _tol

pytestmark = pytest.mark.gpu


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device())


@pytest.mark.parametrize("name", ["f32", "f64"])
def test_bin_keys_from_reference_fold(name):
    """The sort's bin keys equal those derived from the reference's own
    fold_rescale output (i0 = ceil(fold - ns/2), spread.py:214), bit for bit."""
    d = dict(np.load(GOLDEN / "ref_fold.npz"))
    x = d[f"x_{name}"]
    ns = 8
    for nf in (1024, 250):
        fold = d[f"fold_{name}_{nf}"]
        i0 = np.mod(np.ceil(fold - fold.dtype.type(ns / 2.0)).astype(np.int64), nf)
        kp = nb.KernelParams(ns, 2.3 * ns, 4.0 / ns**2, 2.0)
        ps = PointSort([to_dev(x)], (nf,), kp, prenorm=True, tile=(32,))
        keys, _, _ = ps.results()
        assert np.array_equal(keys.cpu().numpy(), i0 // 32)


@pytest.mark.parametrize("kind", [1, 2])
def test_types_1_2_against_reference(kind):
    d, keys = _cases(f"ref_t{kind}.npz")
    for k in keys:
        dim, nm, M, prec, eps, isign, uf, nt = _parse(k)
        dim, eps, isign, uf = int(dim), float(eps), int(isign), float(uf)
        n_modes = tuple(int(v) for v in nm.split("x") if v)
        X = [to_dev(d[f"{k}/x{i}"]) for i in range(dim)]
        if kind == 1:
            fn = {1: nb.nufft1d1, 2: nb.nufft2d1, 3: nb.nufft3d1}[dim]
            out = fn(*X, to_dev(d[f"{k}/c"]), n_modes[0] if dim == 1 else n_modes, eps=eps, isign=isign,
                     upsampfac=uf)
        else:
            fn = {1: nb.nufft1d2, 2: nb.nufft2d2, 3: nb.nufft3d2}[dim]
            out = fn(*X, to_dev(d[f"{k}/f"]), eps=eps, isign=-isign, upsampfac=uf)
        out = out.cpu().numpy()
        ref = d[f"{k}/out"]
        assert out.shape == ref.shape
        tol = 2 * eps if prec == "c128" else _tol(prec, eps, uf)
        assert rel_l2(out, ref) <= tol, k


def test_type3_against_reference():
    d, keys = _cases("ref_t3.npz")
    for k in keys:
        dim, M, K, S, prec, eps, isign, nt = _parse(k)
        dim, eps, isign = int(dim), float(eps), int(isign)
        src = [to_dev(d[f"{k}/x{i}"]) for i in range(dim)]
        tgt = [to_dev(d[f"{k}/s{i}"]) for i in range(dim)]
        nf = [int(v) for v in d[f"{k}/nf"]]
        c = to_dev(d[f"{k}/c"])
        if dim == 1:
            out = nb.nufft1d3(src[0], c, tgt[0], nf[0], eps=eps, isign=isign)
        elif dim == 2:
            out = nb.nufft2d3(*src, c, *tgt, nf, eps=eps, isign=isign)
        else:
            out = nb.nufft3d3(*src, c, *tgt, nf, eps=eps, isign=isign)
        assert rel_l2(out.cpu().numpy(), d[f"{k}/out"]) <= 2 * eps, k


@pytest.mark.parametrize("dim", [2, 3])
def test_core_and_backward_rules_against_reference(dim):
    d = dict(np.load(GOLDEN / "ref_core.npz"))
    p = f"d{dim}"
    ns, beta, c, uf = d["kp"]
    kp = nb.KernelParams(int(ns), float(beta), float(c), float(uf))
    nf = tuple(int(v) for v in d[f"{p}/nf"])
    sp, it = (spread_2d, interp_2d) if dim == 2 else (spread_3d, interp_3d)
    # spread and its backward rule (dx, dy, [dz], dc) for the grid cotangent g
    X = [to_dev(d[f"{p}/x{i}"]).requires_grad_(True) for i in range(dim)]
    cc = to_dev(d[f"{p}/c"]).requires_grad_(True)
    out = sp(*X, cc, *nf, kp)
    assert rel_l2(out.detach().cpu().numpy(), d[f"{p}/spread"]) < 1e-12
    out.backward(to_dev(d[f"{p}/g"]))
    for i in range(dim):
        assert rel_l2(X[i].grad.cpu().numpy(), d[f"{p}/spread_bwd_x{i}"]) < 1e-12
    assert rel_l2(cc.grad.cpu().numpy(), d[f"{p}/spread_bwd_c"]) < 1e-12
    # interp and its backward rule (dx, dy, [dz], dfw) for the point cotangent gp
    X = [to_dev(d[f"{p}/x{i}"]).requires_grad_(True) for i in range(dim)]
    v = it(*[x.detach() for x in X], to_dev(d[f"{p}/fw"]), *nf, kp)
    assert rel_l2(v.cpu().numpy(), d[f"{p}/interp"]) < 1e-12
    fw = to_dev(d[f"{p}/fwr"]).requires_grad_(True)
    it(*X, fw, *nf, kp).backward(to_dev(d[f"{p}/gp"]))
    for i in range(dim):
        assert rel_l2(X[i].grad.cpu().numpy(), d[f"{p}/interp_bwd_x{i}"]) < 1e-12
    assert rel_l2(fw.grad.cpu().numpy(), d[f"{p}/interp_bwd_fw"]) < 1e-12
