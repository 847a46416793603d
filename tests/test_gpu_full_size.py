"""GPU parity at the benchmark sizes: the inputs the bench times, checked in full.

Every case runs the CUDA path at its full size and is checked three ways:

  * the bin sort bit-exact against the oracle (keys, permutation, bin starts);
  * the transform against the oracle (the NumPy restatement of nufftax's
    pure-JAX path), relative l2 <= 2 eps.  Where the oracle cannot run at full
    size in seconds (8 M 3D points: 4 G kernel terms), linearity keeps the GPU
    run at full size while the oracle sees a subset: a type 1 with strengths
    zero outside a random subset S of the points equals the type 1 of S alone
    (a zero strength adds exact zeros), and a type 2 is compared at a subset of
    its targets;
  * against the FP64 direct sum (tests/conftest.py:154-198 of nufftax): type 1
    on 256 modes (a product set, all points), type 2 at 256 targets (all modes).
    The complex64 bound is 10 eps + 2 N 2^-24: coordinates are folded in
    float32, as nufftax folds them, which moves a point's grid position by up
    to 2^-24 of a period and the phase of mode k by up to about k 2^-24 (the
    oracle shows the same error against the direct sum; it is asserted too).

The measured figures are printed (run with -s to see them).
"""

import numpy as np
import pytest
import torch

import bench
import nufftax_b200 as nb
from nufftax_b200 import PointSort
from nufftax_b200.batch import BatchPlan
from oracle import nufft_oracle as O
from tests.conftest import cuda_device, rel_l2

pytestmark = pytest.mark.gpu

EPS = 1e-6


def dev():
    return cuda_device()


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev())


def direct_bound(eps, n_modes, c64=True):
    return 10 * eps + (2 * max(n_modes) * 2.0 ** -24 if c64 else 0.0)


def mode_axes(rng, n_modes, per_axis):
    return [np.sort(rng.choice(np.arange(-(n // 2), (n - 1) // 2 + 1), k, replace=False))
            for n, k in zip(n_modes, per_axis)]


def sub_of(f, axes, n_modes):
    """f (n_d..n_1, CMCL) at the product set of modes `axes` (x first)."""
    idx = [a + n // 2 for a, n in zip(axes, n_modes)]
    return f[np.ix_(*reversed(idx))]


def check_sort(X, nf, kp):
    ps = PointSort([to_dev(x) for x in X], nf, kp, prenorm=True)
    keys, perm, bstart = ps.results()
    okeys, ocells = O.bin_keys(X, nf, kp.nspread, ps.tile, True)
    nbins = int(np.prod([-(-n // t) for n, t in zip(nf, ps.tile)]))
    operm, obs = O.bin_sort(okeys, ocells, nbins, int(np.prod(ps.tile)))
    assert np.array_equal(keys.cpu().numpy(), okeys)
    assert np.array_equal(perm.cpu().numpy(), operm)
    assert np.array_equal(bstart.cpu().numpy(), obs)


# ---------------------------------------------------------------------------
# 2D: the bench's two point sets (radial 524,288 and clustered 4,000,000 on 512^2)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["radial", "clustered"])
def test_bench2d_full_size(name):
    s = [q for q in bench.workload(seed=1234) if q["name"] == name][0]
    X = [s["x"], s["y"]]
    kp = nb.compute_kernel_params(EPS)
    nf = tuple(nb.compute_grid_size(n, 2.0, kp.nspread) for n in bench.N_MODES)
    check_sort(X, nf, kp)
    xd, yd = to_dev(s["x"]), to_dev(s["y"])
    nb.sort_cache.clear()
    f1 = nb.nufft2d1(xd, yd, to_dev(s["c"]), bench.N_MODES, eps=EPS).cpu().numpy()
    c2 = nb.nufft2d2(xd, yd, to_dev(s["f"]), eps=EPS).cpu().numpy()
    r1 = O.nufft_type1(X, s["c"], bench.N_MODES, eps=EPS)
    r2 = O.nufft_type2(X, s["f"], eps=EPS)
    rng = np.random.default_rng(5)
    ax = mode_axes(rng, bench.N_MODES, (16, 16))
    d1 = O.direct_type1_product(X, s["c"], ax, isign=1)
    rows = np.sort(rng.choice(s["M"], 256, replace=False))
    d2 = O.direct_type2_points([s["x"][rows], s["y"][rows]], s["f"], isign=-1)
    e = {"t1_oracle": rel_l2(f1, r1), "t2_oracle": rel_l2(c2, r2), "t1_direct": rel_l2(sub_of(f1, ax, bench.N_MODES), d1),
         "t2_direct": rel_l2(c2[rows], d2), "oracle_t1_direct": rel_l2(sub_of(r1, ax, bench.N_MODES), d1),
         "oracle_t2_direct": rel_l2(r2[rows], d2)}
    print(name, {k: f"{v:.2e}" for k, v in e.items()})
    assert e["t1_oracle"] <= 2 * EPS and e["t2_oracle"] <= 2 * EPS
    bound = direct_bound(EPS, bench.N_MODES)
    assert max(e["t1_direct"], e["t2_direct"], e["oracle_t1_direct"], e["oracle_t2_direct"]) < bound


# ---------------------------------------------------------------------------
# 3D: 8,000,000 uniform points, 128^3 modes (nf 256^3; the plane-owner spread)
# ---------------------------------------------------------------------------
def test_uniform3d_full_size():
    M, N = 8_000_000, (128, 128, 128)
    rng = np.random.default_rng(4)
    X = [rng.uniform(-np.pi, np.pi, M).astype(np.float32) for _ in range(3)]
    c = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    f = (rng.standard_normal(N[::-1]) + 1j * rng.standard_normal(N[::-1])).astype(np.complex64)
    kp = nb.compute_kernel_params(EPS)
    nf = tuple(nb.compute_grid_size(n, 2.0, kp.nspread) for n in N)
    check_sort(X, nf, kp)
    Xd = [to_dev(x) for x in X]
    nb.sort_cache.clear()
    f1 = nb.nufft3d1(*Xd, to_dev(c), N, eps=EPS).cpu().numpy()
    c2 = nb.nufft3d2(*Xd, to_dev(f), eps=EPS).cpu().numpy()
    # oracle: strengths on a subset S only (the GPU still sorts and spreads all M points)
    S = np.sort(rng.choice(M, 200_000, replace=False))
    cS = np.zeros_like(c)
    cS[S] = c[S]
    f1S = nb.nufft3d1(*Xd, to_dev(cS), N, eps=EPS).cpu().numpy()
    r1S = O.nufft_type1([x[S] for x in X], c[S], N, eps=EPS)
    r2S = O.nufft_type2([x[S] for x in X], f, eps=EPS)
    ax = mode_axes(rng, N, (8, 8, 4))
    d1 = O.direct_type1_product(X, c, ax, isign=1)
    rows = np.sort(rng.choice(M, 256, replace=False))
    d2 = O.direct_type2_points([x[rows] for x in X], f, isign=-1)
    e = {"t1_oracle_subset": rel_l2(f1S, r1S), "t2_oracle_subset": rel_l2(c2[S], r2S),
         "t1_direct": rel_l2(sub_of(f1, ax, N), d1), "t2_direct": rel_l2(c2[rows], d2)}
    print("uniform3d", {k: f"{v:.2e}" for k, v in e.items()})
    assert e["t1_oracle_subset"] <= 2 * EPS and e["t2_oracle_subset"] <= 2 * EPS
    assert max(e["t1_direct"], e["t2_direct"]) < direct_bound(EPS, N)


# ---------------------------------------------------------------------------
# Batched: the bench's 64 uneven problems at eps 1e-5 in one graph-captured plan
# ---------------------------------------------------------------------------
def test_batched_full_size():
    eps = 1e-5
    probs = bench.batched_workload()
    d = dev()
    pts = [[to_dev(q["x"]), to_dev(q["y"])] for q in probs]
    plan = BatchPlan(pts, [q["n_modes"] for q in probs], eps=eps, graph=True)
    cs = [to_dev(q["c"]) for q in probs]
    fs = [to_dev(q["f"]) for q in probs]
    f_out, c_out = plan.run(cs, fs)
    f_out = [t.cpu().numpy() for t in f_out]
    c_out = [t.cpu().numpy() for t in c_out]
    worst_plain = 0.0
    for p, q in enumerate(probs):
        nb.sort_cache.clear()
        r1 = nb.nufft2d1(*pts[p], cs[p], q["n_modes"], eps=eps).cpu().numpy()
        r2 = nb.nufft2d2(*pts[p], fs[p], eps=eps).cpu().numpy()
        worst_plain = max(worst_plain, rel_l2(f_out[p], r1), rel_l2(c_out[p], r2))
    # oracle and direct sum on eight problems (the four largest and four smallest,
    # uniform and clustered), strengths kept on a subset for the oracle's type 1
    rng = np.random.default_rng(9)
    order = np.argsort([q["M"] for q in probs])
    chosen = list(order[:4]) + list(order[-4:])
    masked = []
    for p, q in enumerate(probs):
        cm = np.zeros_like(q["c"])
        if p in chosen:
            S = np.sort(rng.choice(q["M"], min(q["M"], 100_000), replace=False))
            cm[S] = q["c"][S]
            masked.append(S)
        else:
            masked.append(None)
        plan.c_in[p].copy_(to_dev(cm))
    f_m, _ = plan.run()
    worst = {"t1_oracle_subset": 0.0, "t2_oracle_subset": 0.0, "t1_direct": 0.0, "t2_direct": 0.0}
    for p in chosen:
        q = probs[p]
        X = [q["x"], q["y"]]
        S = masked[p]
        r1 = O.nufft_type1([x[S] for x in X], q["c"][S], q["n_modes"], eps=eps)
        worst["t1_oracle_subset"] = max(worst["t1_oracle_subset"], rel_l2(f_m[p].cpu().numpy(), r1))
        rows = np.sort(rng.choice(q["M"], min(q["M"], 20_000), replace=False))
        r2 = O.nufft_type2([x[rows] for x in X], q["f"], eps=eps)
        worst["t2_oracle_subset"] = max(worst["t2_oracle_subset"], rel_l2(c_out[p][rows], r2))
        ax = mode_axes(rng, q["n_modes"], (16, 16))
        d1 = O.direct_type1_product(X, q["c"], ax, isign=1)
        worst["t1_direct"] = max(worst["t1_direct"], rel_l2(sub_of(f_out[p], ax, q["n_modes"]), d1))
        d2 = O.direct_type2_points([x[rows[:256]] for x in X], q["f"], isign=-1)
        worst["t2_direct"] = max(worst["t2_direct"], rel_l2(c_out[p][rows[:256]], d2))
    print("batched", f"plain {worst_plain:.2e}", {k: f"{v:.2e}" for k, v in worst.items()})
    assert worst_plain <= 2 * eps
    assert worst["t1_oracle_subset"] <= 2 * eps and worst["t2_oracle_subset"] <= 2 * eps
    assert max(worst["t1_direct"], worst["t2_direct"]) < direct_bound(eps, (512, 512))


# ---------------------------------------------------------------------------
# Type 3 at the served geometry: sources in [-pi, pi)^2, targets in [-300, 300]^2
# (type-3 grid 1250^2, inner type 2 on 2500^2), M = K = 1,000,000
# ---------------------------------------------------------------------------
def test_type3_served_geometry():
    M = K = 1_000_000
    rng = np.random.default_rng(31)
    src = [rng.uniform(-np.pi, np.pi, M) for _ in range(2)]
    tgt = [rng.uniform(-300.0, 300.0, K) for _ in range(2)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    nf = nb.compute_type3_grid_sizes_2d(np.pi, np.pi, 300.0, 300.0, eps=EPS)
    assert tuple(nf) == (1250, 1250)
    rows = np.sort(rng.choice(K, 256, replace=False))
    direct = O.direct_type3(src, c, [t[rows] for t in tgt], isign=1)
    e = {}
    # complex128 against the oracle on the same float64 inputs
    f128 = nb.nufft2d3(*[to_dev(a) for a in src], to_dev(c), *[to_dev(a) for a in tgt], nf, eps=EPS).cpu().numpy()
    ref = O.nufft_type3(src, c, tgt, nf, eps=EPS, isign=1)
    e["c128_oracle"] = rel_l2(f128, ref)
    e["c128_direct"] = rel_l2(f128[rows], direct)
    # complex64: the oracle on the float32-rounded inputs (it computes in float64,
    # so the difference is this path's float32 arithmetic)
    s32 = [a.astype(np.float32) for a in src]
    t32 = [a.astype(np.float32) for a in tgt]
    c64 = c.astype(np.complex64)
    f64 = nb.nufft2d3(*[to_dev(a) for a in s32], to_dev(c64), *[to_dev(a) for a in t32], nf, eps=EPS).cpu().numpy()
    ref32 = O.nufft_type3(s32, c64, t32, nf, eps=EPS, isign=1)
    e["c64_oracle_f32_inputs"] = rel_l2(f64, ref32)
    e["c64_direct"] = rel_l2(f64[rows], direct)
    ref32_direct = rel_l2(ref32[rows], direct)
    print("type3 served", {k: f"{v:.2e}" for k, v in e.items()}, f"oracle_c64_direct {ref32_direct:.2e}")
    assert e["c128_oracle"] <= 2 * EPS
    assert e["c128_direct"] < 10 * EPS
    # complex64 against the oracle on the same float32 inputs, which follows the
    # reference's float32 rescaling of sources and targets: 2 eps
    assert e["c64_oracle_f32_inputs"] <= 2 * EPS
    # against the exact sum, complex64 carries the float32 fold of the targets
    # on the inner grid of the type-3 grid's modes (nf = 1250 per axis), as the
    # reference does: 10 eps + 2 nf 2^-24, the oracle's own error included
    bound = direct_bound(EPS, nf)
    assert e["c64_direct"] < bound and ref32_direct < bound
