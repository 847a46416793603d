"""CPU: the oracle against golden vectors computed by the reference's own source.

tests/golden/ref_*.npz come from make_reference_golden.py, which runs
nufftax's pure-JAX modules unmodified on NumPy through jax_numpy_shim.py (in
the reference tests' x64 configuration).  These tests pin the oracle to them:

  * coordinate pre-normalisation and fold_rescale: bit-exact (float32 and
    float64, folding edge cases included);
  * transforms, core spread / interp and the custom_vjp backward rules:
    complex128 to 1e-12 relative (both sides compute in float64); complex64
    inputs within 2 eps (the reference accumulates complex64 in float32, the
    oracle in float64; type 3 follows the reference's float32 rescaling).
"""

import numpy as np
import pytest

from oracle import nufft_oracle as O
from tests.conftest import GOLDEN, rel_l2


def _cases(name):
    d = dict(np.load(GOLDEN / name))
    keys = sorted({k.split("/")[0] for k in d if "/" in k})
    return d, keys


def _parse(key):
    parts = key.split("_")
    return parts


def test_fold_and_premod_bit_exact():
    d = dict(np.load(GOLDEN / "ref_fold.npz"))
    for name in ("f32", "f64"):
        x = d[f"x_{name}"]
        pre = O.premod(x)
        assert pre.dtype == x.dtype
        assert np.array_equal(pre, d[f"premod_{name}"])
        for nf in (16384, 1024, 250, 7):
            assert np.array_equal(O.fold_rescale(pre, nf), d[f"fold_{name}_{nf}"])


def _tol(prec, eps, uf=2.0, c128=1e-12):
    if prec == "c128":
        return c128
    # complex64: 2 eps; at upsampfac 1.25 the deconvolution factors are larger
    # and amplify the reference's own float32 accumulation to ~3e-6 against
    # float64 arithmetic (the oracle matches it to 1e-16 in float64 there):
    # 5 eps.  The reference itself is 4.4e-5 from the exact sum at 1.25
    # (tests/test_upsampfac.py only asserts 1e-2).
    return 2 * eps if uf == 2.0 else 5 * eps


@pytest.mark.parametrize("kind", [1, 2])
def test_types_1_2_against_reference(kind):
    d, keys = _cases(f"ref_t{kind}.npz")
    assert len(keys) == 7
    for k in keys:
        dim, nm, M, prec, eps, isign, uf, nt = _parse(k)
        dim, eps, isign, uf = int(dim), float(eps), int(isign), float(uf)
        n_modes = tuple(int(v) for v in nm.split("x") if v)
        X = [d[f"{k}/x{i}"] for i in range(dim)]
        if kind == 1:
            out = O.nufft_type1(X, d[f"{k}/c"], n_modes, eps=eps, isign=isign, upsampfac=uf)
        else:
            out = O.nufft_type2(X, d[f"{k}/f"], eps=eps, isign=-isign, upsampfac=uf)
        assert out.shape == d[f"{k}/out"].shape
        assert rel_l2(out, d[f"{k}/out"]) <= _tol(prec, eps, uf), k


def test_type3_against_reference():
    d, keys = _cases("ref_t3.npz")
    assert len(keys) == 4
    for k in keys:
        dim, M, K, S, prec, eps, isign, nt = _parse(k)
        dim, eps, isign = int(dim), float(eps), int(isign)
        src = [d[f"{k}/x{i}"] for i in range(dim)]
        tgt = [d[f"{k}/s{i}"] for i in range(dim)]
        out = O.nufft_type3(src, d[f"{k}/c"], tgt, list(d[f"{k}/nf"]), eps=eps, isign=isign)
        assert rel_l2(out, d[f"{k}/out"]) <= _tol(prec, eps), k


@pytest.mark.parametrize("dim", [2, 3])
def test_core_spread_interp_and_backward_rules(dim):
    d = dict(np.load(GOLDEN / "ref_core.npz"))
    p = f"d{dim}"
    ns, beta, c, uf = d["kp"]
    kp = O.KernelParams(int(ns), float(beta), float(c), float(uf))
    X = [d[f"{p}/x{i}"] for i in range(dim)]
    nf = tuple(int(v) for v in d[f"{p}/nf"])
    assert rel_l2(O.spread(X, d[f"{p}/c"], nf, kp), d[f"{p}/spread"]) < 1e-12
    assert rel_l2(O.interp(X, d[f"{p}/fw"], kp), d[f"{p}/interp"]) < 1e-12
    gs = O.spread_grad_coords(X, d[f"{p}/c"], d[f"{p}/g"], kp)
    gi = O.interp_grad_coords(X, d[f"{p}/fwr"], d[f"{p}/gp"], kp)
    for i in range(dim):
        assert rel_l2(gs[i], d[f"{p}/spread_bwd_x{i}"]) < 1e-12
        assert rel_l2(gi[i], d[f"{p}/interp_bwd_x{i}"]) < 1e-12
    # dc of spread is interp(g); dfw of interp is spread(g) (spread.py:983-990)
    assert rel_l2(O.interp(X, d[f"{p}/g"], kp), d[f"{p}/spread_bwd_c"]) < 1e-12
    assert rel_l2(O.spread(X, d[f"{p}/gp"], nf, kp), d[f"{p}/interp_bwd_fw"]) < 1e-12
