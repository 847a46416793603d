"""GPU: batched plans (one persistent launch over many uneven problems, CUDA graph).

Each problem's batched result must equal the plain per-problem path within the
transform tolerance (relative l2 <= 2 eps against the oracle), with and without
graph capture, over repeated runs with changing inputs.
"""

import numpy as np
import pytest
import torch

import nufftax_b200 as nb
from nufftax_b200.autotune import tune
from nufftax_b200.batch import BatchPlan
from oracle import nufft_oracle as O
from tests.conftest import cuda_device, rel_l2

pytestmark = pytest.mark.gpu


def _problems(rng, dim, P, eps):
    dev = cuda_device()
    pts, modes = [], []
    sizes = [16, 24, 40, 64] if dim == 2 else [8, 12, 16]
    for p in range(P):
        M = int(rng.integers(200, 20000))
        if p % 2:
            X = [np.mod(0.3 * rng.standard_normal(M) + np.pi, 2 * np.pi) - np.pi for _ in range(dim)]
        else:
            X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        pts.append([torch.from_numpy(x.astype(np.float32)).to(dev) for x in X])
        modes.append(tuple(int(rng.choice(sizes)) for _ in range(dim)))
    return pts, modes


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_plain(dim, graph):
    rng = np.random.default_rng(10 + dim)
    eps = 1e-5
    pts, modes = _problems(rng, dim, 9, eps)
    plan = BatchPlan(pts, modes, eps=eps, graph=graph)
    dev = cuda_device()
    for rep in range(3):
        cs = [torch.from_numpy((rng.standard_normal(m) + 1j * rng.standard_normal(m)).astype(np.complex64)).to(dev)
              for m in plan.M]
        fs = [torch.from_numpy((rng.standard_normal(tuple(reversed(nm))) + 1j * rng.standard_normal(
            tuple(reversed(nm)))).astype(np.complex64)).to(dev) for nm in modes]
        f_out, c_out = plan.run(cs, fs)
        for p in range(plan.P):
            t1 = {2: nb.nufft2d1, 3: nb.nufft3d1}[dim]
            t2 = {2: nb.nufft2d2, 3: nb.nufft3d2}[dim]
            ref1 = t1(*pts[p], cs[p], modes[p], eps=eps)
            ref2 = t2(*pts[p], fs[p], eps=eps)
            assert rel_l2(f_out[p].cpu().numpy(), ref1.cpu().numpy()) <= 2 * eps
            assert rel_l2(c_out[p].cpu().numpy(), ref2.cpu().numpy()) <= 2 * eps
        if rep == 0:
            # one problem against the oracle directly
            X = [t.cpu().numpy() for t in pts[1]]
            ref = O.nufft_type1(X, cs[1].cpu().numpy(), modes[1], eps=eps)
            assert rel_l2(f_out[1].cpu().numpy(), ref) <= 2 * eps


def test_batch_points_updated_in_place():
    rng = np.random.default_rng(7)
    dev = cuda_device()
    pts, modes = _problems(rng, 2, 4, 1e-6)
    plan = BatchPlan(pts, modes, eps=1e-6, graph=True)
    cs = [torch.ones(m, dtype=torch.complex64, device=dev) for m in plan.M]
    plan.run(cs, None)
    # move the points: the captured sort re-reads them
    for p in range(plan.P):
        for t in plan.points[p]:
            t.copy_(torch.from_numpy(rng.uniform(-np.pi, np.pi, t.numel()).astype(np.float32)).to(dev))
    f_out, _ = plan.run(cs, None)
    for p in range(plan.P):
        ref = nb.nufft2d1(*plan.points[p], cs[p], modes[p], eps=1e-6)
        assert rel_l2(f_out[p].cpu().numpy(), ref.cpu().numpy()) <= 2e-6


def test_autotune_returns_valid_tiling():
    rng = np.random.default_rng(3)
    dev = cuda_device()
    x, y = [torch.from_numpy(rng.uniform(-np.pi, np.pi, 50000).astype(np.float32)).to(dev) for _ in range(2)]
    kp = nb.compute_kernel_params(1e-5)
    timings = []
    tile, maxsub, modes = tune([x, y], (256, 256), kp, timings=timings)
    assert len(tile) == 2 and maxsub > 0 and len(modes) == 2
    # both threads-per-point modes of the 2D interpolation were timed
    assert {m[1] for _, _, _, m in timings} == {nb._lib.NFX_PER_POINT_THREAD, nb._lib.NFX_PER_POINT_GROUP}
    # the tuned choice gives the same spread and interpolation
    ps_a = nb.PointSort([x, y], (256, 256), kp, prenorm=True, tile=tile, max_subproblem=maxsub, modes=modes)
    ps_b = nb.PointSort([x, y], (256, 256), kp, prenorm=True)
    c = torch.ones((1, 50000), dtype=torch.complex64, device=dev)
    fa, fb = ps_a.spread(c), ps_b.spread(c)
    assert rel_l2(fa.cpu().numpy(), fb.cpu().numpy()) < 2e-6
    assert rel_l2(ps_a.interp(fa).cpu().numpy(), ps_b.interp(fb).cpu().numpy()) < 2e-6
    assert tune([x, y], (256, 256), kp) == (tile, maxsub, modes)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("prec", ["c64", "c128"])
def test_threads_per_point_modes_agree_with_oracle(dim, prec):
    """Every threads-per-point mode of spread and interpolation (one thread /
    lane group per point; one warp / the CTA per point) matches the oracle."""
    from oracle import nufft_oracle as O

    rng = np.random.default_rng(30 + dim)
    dev = cuda_device()
    rdt, cdt = (np.float32, np.complex64) if prec == "c64" else (np.float64, np.complex128)
    tol = 2e-6 if prec == "c64" else 1e-12
    kp = nb.compute_kernel_params(1e-6 if prec == "c64" else 1e-12)
    nf = (64, 48) if dim == 2 else (32, 24, 20)
    M = 20000
    X = [rng.uniform(-np.pi, np.pi, M).astype(rdt) for _ in range(dim)]
    c = (rng.standard_normal((1, M)) + 1j * rng.standard_normal((1, M))).astype(cdt)
    g = (rng.standard_normal((1,) + nf[::-1]) + 1j * rng.standard_normal((1,) + nf[::-1])).astype(cdt)
    ref_s = O.spread(X, c, nf, kp)
    ref_i = O.interp(X, g, kp)
    L = nb._lib
    spread_modes = [L.NFX_PER_POINT_WARP] + ([L.NFX_PER_POINT_CTA] if dim == 3 else [])
    for sm in spread_modes:
        for im in (L.NFX_PER_POINT_THREAD, L.NFX_PER_POINT_GROUP):
            ps = nb.PointSort([torch.from_numpy(x).to(dev) for x in X], nf, kp, prenorm=False, modes=(sm, im))
            fw = ps.spread(torch.from_numpy(c).to(dev)).cpu().numpy()
            ci = ps.interp(torch.from_numpy(g).to(dev)).cpu().numpy()
            assert rel_l2(fw, ref_s) < tol, (sm, im)
            assert rel_l2(ci, ref_i) < tol, (sm, im)
