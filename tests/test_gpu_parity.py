"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Tolerances (written per test):
  * bin keys, permutation and bin offsets: bit-exact;
  * transforms: relative l2 <= 2 eps against the oracle's restatement of
    nufftax's pure-JAX path (complex64 for eps >= 1e-6, complex128 below), and
    the error against the FP64 direct sum on a subsample is asserted < 10 eps
    (the bar nufftax's own tests use against an exact transform) plus, for
    complex64, 2 N 2^-24: the reference folds coordinates in float32, so a
    point's grid position carries a relative rounding of 2^-24, i.e. a phase
    error up to about N 2^-24 at the highest of N modes;
  * spread / interp components: relative l2 <= 2e-6 (complex64) or 1e-12
    (complex128) against the oracle's float64 accumulation.
"""

import numpy as np
import pytest
import torch

import nufftax_b200 as nb
from nufftax_b200 import PointSort
from nufftax_b200.core import interp_1d, interp_2d, interp_3d, spread_1d, spread_2d, spread_3d
from oracle import nufft_oracle as O
from tests.conftest import GOLDEN, cuda_device, rel_l2

pytestmark = pytest.mark.gpu


def dev():
    return cuda_device()


def to_dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(dev())
    return t if dtype is None else t.to(dtype)


def rand_c(rng, shape, dtype=np.complex64):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


# ---------------------------------------------------------------------------
# Sort: bit-exact
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["sort_1d", "sort_2d", "sort_3d"])
@pytest.mark.parametrize("prenorm", [0, 1])
def test_sort_golden_bit_exact(name, prenorm):
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    dim = len(d["nf"])
    X = [to_dev(d[f"x{i}"]) for i in range(dim)]
    ns = int(d["ns"])
    kp = nb.KernelParams(ns, 2.3 * ns, 4.0 / ns**2, 2.0)
    ps = PointSort(X, tuple(int(v) for v in d["nf"]), kp, bool(prenorm), tile=tuple(int(v) for v in d["tile"]))
    keys, perm, bstart = ps.results()
    assert np.array_equal(keys.cpu().numpy(), d[f"keys_p{prenorm}"])
    assert np.array_equal(perm.cpu().numpy(), d[f"perm_p{prenorm}"])
    assert np.array_equal(bstart.cpu().numpy(), d[f"bin_start_p{prenorm}"])


@pytest.mark.parametrize("dim,nf,dist", [(1, (16384,), "uniform"), (2, (1024, 1024), "uniform"),
                                         (2, (1024, 1024), "cluster"), (3, (128, 96, 64), "uniform"),
                                         (2, (256, 256), "onecell")])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_sort_random_bit_exact(dim, nf, dist, dtype):
    rng = np.random.default_rng(7)
    M = 200_003
    if dist == "uniform":
        X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
    elif dist == "cluster":
        X = [np.mod(0.3 * rng.standard_normal(M) + np.pi, 2 * np.pi) - np.pi for _ in range(dim)]
    else:
        X = [np.full(M, 0.1234) for _ in range(dim)]
    X = [x.astype(dtype) for x in X]
    kp = nb.compute_kernel_params(1e-6)
    ps = PointSort([to_dev(x) for x in X], nf, kp, prenorm=True)
    keys, perm, bstart = ps.results()
    okeys, ocells = O.bin_keys(X, nf, kp.nspread, ps.tile, True)
    operm, obs = O.bin_sort(okeys, ocells, int(np.prod([-(-n // t) for n, t in zip(nf, ps.tile)])),
                            int(np.prod(ps.tile)))
    assert np.array_equal(keys.cpu().numpy(), okeys)
    assert np.array_equal(perm.cpu().numpy(), operm)
    assert np.array_equal(bstart.cpu().numpy(), obs)


def test_sort_empty_and_single():
    kp = nb.compute_kernel_params(1e-6)
    for M in (0, 1):
        X = [to_dev(np.full(M, 0.5, np.float32)) for _ in range(2)]
        ps = PointSort(X, (64, 64), kp, prenorm=True)
        _, perm, bstart = ps.results()
        assert perm.numel() == M
        assert int(bstart[-1]) == M


# ---------------------------------------------------------------------------
# Spread / interp components
# ---------------------------------------------------------------------------
# The 3D cases cover both 3D spreads: fewer points than grid cells (plane-owner
# spread) and more (run-merging spread).
CASES = [(1, (64,), 700), (1, (1000,), 3000), (2, (48, 40), 2000), (2, (256, 192), 20000), (3, (24, 20, 32), 4000),
         (3, (12, 10, 16), 6000)]


@pytest.mark.parametrize("dim,nf,M", CASES)
@pytest.mark.parametrize("eps", [1e-2, 1e-6, 1e-12, 1e-15])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_spread_interp_vs_oracle(dim, nf, M, eps, prec):
    if prec == "f32" and eps < 1e-7:
        pytest.skip("complex64 is tested at eps >= 1e-6")
    rng = np.random.default_rng(11 + dim)
    rdt, cdt = (np.float32, np.complex64) if prec == "f32" else (np.float64, np.complex128)
    tol = 2e-6 if prec == "f32" else 1e-12
    kp = nb.compute_kernel_params(eps)
    X = [rng.uniform(-np.pi, np.pi, M).astype(rdt) for _ in range(dim)]
    c = rand_c(rng, (2, M), cdt)
    Xd = [to_dev(x) for x in X]
    fns = {1: (spread_1d, interp_1d), 2: (spread_2d, interp_2d), 3: (spread_3d, interp_3d)}[dim]
    fw = fns[0](*Xd, to_dev(c), *nf, kp).cpu().numpy()
    ref = O.spread(X, c, nf, kp)
    assert fw.shape == ref.shape
    assert rel_l2(fw, ref) < tol
    g = rand_c(rng, (2,) + tuple(reversed(nf)), cdt)
    ci = fns[1](*Xd, to_dev(g), *nf, kp).cpu().numpy()
    assert rel_l2(ci, O.interp(X, g, kp)) < tol


@pytest.mark.parametrize("ns_eps", [1e-1, 1e-3, 1e-5, 1e-7, 1e-9, 1e-11, 1e-13, 1e-15])
def test_every_kernel_width_3d_float_owner(ns_eps):
    """3D complex64 spread with fewer points than cells (the plane-owner kernel and
    its 16-byte staging slots) at every even nspread, against the oracle; float
    weights and sums bound the error near 1e-6 whatever the width."""
    rng = np.random.default_rng(5)
    kp = nb.compute_kernel_params(ns_eps)
    nf, M = (36, 34, 40), 1500
    X = [rng.uniform(-np.pi, np.pi, M).astype(np.float32) for _ in range(3)]
    c = rand_c(rng, M, np.complex64)
    fw = spread_3d(*[to_dev(x) for x in X], to_dev(c), *nf, kp).cpu().numpy()
    assert rel_l2(fw, O.spread(X, c, nf, kp)) < 1e-5


@pytest.mark.parametrize("ns_eps", [1e-1, 1e-3, 1e-5, 1e-7, 1e-9, 1e-11, 1e-13, 1e-15])
def test_every_kernel_width(ns_eps):
    """Every even nspread 2..16 compiles, launches and matches (complex128)."""
    rng = np.random.default_rng(3)
    kp = nb.compute_kernel_params(ns_eps)
    for dim, nf in ((1, (80,)), (2, (40, 36)), (3, (36, 34, 40))):
        M = 1500
        X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        c = rand_c(rng, M, np.complex128)
        fn = {1: spread_1d, 2: spread_2d, 3: spread_3d}[dim]
        fw = fn(*[to_dev(x) for x in X], to_dev(c), *nf, kp).cpu().numpy()
        assert rel_l2(fw, O.spread(X, c, nf, kp)) < 1e-12


def test_collisions_all_points_in_one_cell():
    """Heavy same-cell collisions (clustered worst case) stay exact."""
    rng = np.random.default_rng(5)
    M = 100_000
    kp = nb.compute_kernel_params(1e-6)
    X = [np.full(M, 0.25, np.float32), np.full(M, -1.0, np.float32)]
    c = rand_c(rng, M)
    fw = spread_2d(*[to_dev(x) for x in X], to_dev(c), 64, 64, kp).cpu().numpy()
    assert rel_l2(fw, O.spread(X, c, (64, 64), kp)) < 2e-6


def test_tiny_grid_wraps_onto_itself():
    """nf smaller than a padded tile: the footprint wraps around the grid."""
    rng = np.random.default_rng(9)
    kp = nb.compute_kernel_params(1e-9)
    X = [rng.uniform(-np.pi, np.pi, 500) for _ in range(2)]
    c = rand_c(rng, 500, np.complex128)
    fw = spread_2d(*[to_dev(x) for x in X], to_dev(c), 20, 22, kp).cpu().numpy()
    assert rel_l2(fw, O.spread(X, c, (20, 22), kp)) < 1e-12


def test_adjoint_identity_gpu():
    rng = np.random.default_rng(42)
    kp = nb.compute_kernel_params(1e-9)
    for dim, nf in ((1, (64,)), (2, (32, 24)), (3, (16, 12, 20))):
        X = [to_dev(rng.uniform(-np.pi, np.pi, 500)) for _ in range(dim)]
        c = to_dev(rand_c(rng, 500, np.complex128))
        g = to_dev(rand_c(rng, tuple(reversed(nf)), np.complex128))
        sp = {1: spread_1d, 2: spread_2d, 3: spread_3d}[dim]
        it = {1: interp_1d, 2: interp_2d, 3: interp_3d}[dim]
        lhs = torch.vdot(sp(*X, c, *nf, kp).flatten(), g.flatten())
        rhs = torch.vdot(c, it(*X, g, *nf, kp))
        assert abs(complex(lhs - rhs)) / abs(complex(lhs)) < 1e-12


# ---------------------------------------------------------------------------
# Transforms
# ---------------------------------------------------------------------------
def direct_tol(eps, prec, n_modes):
    """Bound against the exact sum: 10 eps, plus the float32 fold limit for complex64."""
    return 10 * eps + (2 * max(n_modes) * 2.0**-24 if prec == "c64" else 0.0)


def _sub_modes(rng, n_modes, K=256):
    ks = O.flat_mode_list(n_modes)
    if ks.shape[0] <= K:
        return np.arange(ks.shape[0]), ks
    idx = np.sort(rng.choice(ks.shape[0], K, replace=False))
    return idx, ks[idx]


T12 = [(1, (64,), 1000), (1, (8192,), 20000), (2, (32, 24), 3000), (2, (128, 128), 40000), (3, (16, 12, 10), 3000),
       (3, (32, 32, 32), 30000)]


@pytest.mark.parametrize("dim,n_modes,M", T12)
@pytest.mark.parametrize("eps,prec", [(1e-6, "c64"), (1e-3, "c64"), (1e-9, "c128"), (1e-12, "c128")])
@pytest.mark.parametrize("isign", [1, -1])
def test_type1_parity(dim, n_modes, M, eps, prec, isign):
    rng = np.random.default_rng(100 + dim)
    rdt, cdt = (np.float32, np.complex64) if prec == "c64" else (np.float64, np.complex128)
    X = [rng.uniform(-np.pi, np.pi, M).astype(rdt) for _ in range(dim)]
    c = rand_c(rng, M, cdt)
    fn = {1: nb.nufft1d1, 2: nb.nufft2d1, 3: nb.nufft3d1}[dim]
    nm = n_modes[0] if dim == 1 else n_modes
    f = fn(*[to_dev(x) for x in X], to_dev(c), nm, eps=eps, isign=isign).cpu().numpy()
    ref = O.nufft_type1(X, c, n_modes, eps=eps, isign=isign)
    assert f.dtype == cdt and f.shape == ref.shape
    assert rel_l2(f, ref) <= 2 * eps
    idx, ks = _sub_modes(rng, n_modes)
    direct = O.direct_type1(X, c, n_modes, isign=isign, flat_modes=ks)
    assert rel_l2(f.ravel()[idx], direct) < direct_tol(eps, prec, n_modes)


@pytest.mark.parametrize("dim,n_modes,M", T12)
@pytest.mark.parametrize("eps,prec", [(1e-6, "c64"), (1e-9, "c128"), (1e-12, "c128")])
@pytest.mark.parametrize("isign", [-1, 1])
def test_type2_parity(dim, n_modes, M, eps, prec, isign):
    rng = np.random.default_rng(200 + dim)
    rdt, cdt = (np.float32, np.complex64) if prec == "c64" else (np.float64, np.complex128)
    X = [rng.uniform(-np.pi, np.pi, M).astype(rdt) for _ in range(dim)]
    f = rand_c(rng, tuple(reversed(n_modes)), cdt)
    fn = {1: nb.nufft1d2, 2: nb.nufft2d2, 3: nb.nufft3d2}[dim]
    c = fn(*[to_dev(x) for x in X], to_dev(f), eps=eps, isign=isign).cpu().numpy()
    ref = O.nufft_type2(X, f, eps=eps, isign=isign)
    assert c.dtype == cdt and c.shape == (M,)
    assert rel_l2(c, ref) <= 2 * eps
    rows = rng.choice(M, min(M, 256), replace=False)
    vals, flat = O.modes_as_flat(f, dim)
    direct = O.direct_type2(X, vals, flat, isign=isign, rows=rows)
    assert rel_l2(c[rows], direct) < direct_tol(eps, prec, n_modes)


@pytest.mark.parametrize("name", ["t1_1d", "t1_2d", "t1_3d"])
def test_type1_golden(name):
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    dim = len(d["n_modes"])
    fn = {1: nb.nufft1d1, 2: nb.nufft2d1, 3: nb.nufft3d1}[dim]
    nm = int(d["n_modes"][0]) if dim == 1 else tuple(int(v) for v in d["n_modes"])
    for e in d["eps"]:
        f = fn(*[to_dev(d[f"x{i}"]) for i in range(dim)], to_dev(d["c"]), nm, eps=float(e),
               isign=int(d["isign"])).cpu().numpy()
        assert rel_l2(f, d[f"oracle_{e:g}"]) <= 2 * e
        assert rel_l2(f, d["direct"]) < 10 * e


@pytest.mark.parametrize("name", ["t2_1d", "t2_2d", "t2_3d"])
def test_type2_golden(name):
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    dim = d["f"].ndim
    fn = {1: nb.nufft1d2, 2: nb.nufft2d2, 3: nb.nufft3d2}[dim]
    for e in d["eps"]:
        c = fn(*[to_dev(d[f"x{i}"]) for i in range(dim)], to_dev(d["f"]), eps=float(e),
               isign=int(d["isign"])).cpu().numpy()
        assert rel_l2(c, d[f"oracle_{e:g}"]) <= 2 * e
        assert rel_l2(c, d["direct"]) < 10 * e


@pytest.mark.parametrize("name", ["t3_1d", "t3_2d", "t3_3d"])
@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_type3_golden(name, prec):
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    dim = len(d["nf"])
    rdt, cdt = (np.float32, np.complex64) if prec == "c64" else (np.float64, np.complex128)
    fn = {1: nb.nufft1d3, 2: nb.nufft2d3, 3: nb.nufft3d3}[dim]
    nf = int(d["nf"][0]) if dim == 1 else tuple(int(v) for v in d["nf"])
    src = [to_dev(d[f"x{i}"].astype(rdt)) for i in range(dim)]
    tgt = [to_dev(d[f"s{i}"].astype(rdt)) for i in range(dim)]
    f = fn(*src, to_dev(d["c"].astype(cdt)), *tgt, nf, eps=1e-6).cpu().numpy()
    if prec == "c128":
        assert rel_l2(f, d["oracle_1e-06"]) <= 2e-6
    else:
        # the oracle on the same float32 inputs follows the reference's float32
        # rescaling of sources and targets
        ref = O.nufft_type3([d[f"x{i}"].astype(rdt) for i in range(dim)], d["c"].astype(cdt),
                            [d[f"s{i}"].astype(rdt) for i in range(dim)], list(d["nf"]), eps=1e-6)
        assert rel_l2(f, ref) <= 2e-6
    # tests/test_nufft3.py:48 asserts 1e-4 against the direct sum at eps = 1e-6
    assert rel_l2(f, d["direct"]) < 1e-4


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_type3_parity_c128(dim):
    rng = np.random.default_rng(300 + dim)
    M, K = 3000, 2000
    src = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
    tgt = [rng.uniform(-40, 40, K) for _ in range(dim)]
    c = rand_c(rng, (2, M), np.complex128)
    eps = 1e-9
    nf = [O.type3_grid_size((a.max() - a.min()) / 2, (b.max() - b.min()) / 2, eps) for a, b in zip(src, tgt)]
    fn = {1: nb.nufft1d3, 2: nb.nufft2d3, 3: nb.nufft3d3}[dim]
    f = fn(*[to_dev(a) for a in src], to_dev(c), *[to_dev(a) for a in tgt], nf[0] if dim == 1 else nf,
           eps=eps, isign=-1).cpu().numpy()
    ref = O.nufft_type3(src, c, tgt, nf, eps=eps, isign=-1)
    assert rel_l2(f, ref) <= 2 * eps
    assert rel_l2(f, O.direct_type3(src, c, tgt, isign=-1)) < 10 * eps


def test_batched_and_upsampfac():
    rng = np.random.default_rng(17)
    M = 5000
    x, y = rng.uniform(-np.pi, np.pi, (2, M)).astype(np.float32)
    c = rand_c(rng, (3, M))
    f = nb.nufft2d1(to_dev(x), to_dev(y), to_dev(c), (40, 30), eps=1e-6).cpu().numpy()
    assert f.shape == (3, 30, 40)
    assert rel_l2(f, O.nufft_type1([x, y], c, (40, 30))) <= 2e-6
    g = nb.nufft2d1(to_dev(x), to_dev(y), to_dev(c[1]), (40, 30), eps=1e-6, upsampfac=(2.0, 1.25)).cpu().numpy()
    assert rel_l2(g, f[1]) <= 4e-6
    h = nb.nufft2d1(to_dev(x), to_dev(y), to_dev(c[0]), (40, 30), eps=1e-6, upsampfac=1.25).cpu().numpy()
    # tests/test_upsampfac.py:41-54 only asserts 1e-2 at upsampfac 1.25
    assert rel_l2(h, O.nufft_type1([x, y], c[0], (40, 30), upsampfac=1.25)) <= 1e-5
    assert rel_l2(h, f[0]) < 1e-2


def test_host_arrays_round_trip():
    rng = np.random.default_rng(18)
    x = rng.uniform(-np.pi, np.pi, 1000).astype(np.float32)
    c = rand_c(rng, 1000)
    f = nb.nufft1d1(x, c, 64)
    assert isinstance(f, np.ndarray) and f.dtype == np.complex64
    back = nb.nufft1d2(torch.from_numpy(x), torch.from_numpy(f))
    assert isinstance(back, torch.Tensor) and not back.is_cuda


# -- known answers of the reference's tests/test_edge_cases.py -------------------------------
def test_edge_cases_known_answers():
    d = dev()
    f = nb.nufft1d1(torch.tensor([0.5], device=d), torch.tensor([1 + 1j], dtype=torch.complex64, device=d), 16)
    k = np.arange(-8, 8)
    assert np.allclose(f.cpu().numpy(), (1 + 1j) * np.exp(1j * k * 0.5), rtol=1e-5)
    f = nb.nufft1d1(torch.zeros(10, device=d), torch.ones(10, dtype=torch.complex64, device=d), 32)
    assert np.allclose(f.cpu().numpy(), 10, rtol=1e-5)
    f = nb.nufft1d1(torch.full((10,), np.pi, device=d), torch.ones(10, dtype=torch.complex64, device=d), 32)
    k = np.arange(-16, 16)
    assert np.allclose(f.cpu().numpy(), 10 * np.exp(1j * k * np.pi), rtol=1e-5, atol=1e-4)
    N = 32
    x = torch.linspace(-np.pi, np.pi, N + 1, device=d)[:-1]
    f = nb.nufft1d1(x, torch.ones(N, dtype=torch.complex64, device=d), N).cpu().numpy()
    assert abs(abs(f[N // 2]) - N) < 1e-4 * N
    assert np.max(np.abs(np.delete(f, N // 2))) < 1e-4
    z = nb.nufft2d1(torch.rand(100, device=d), torch.rand(100, device=d), torch.zeros(100, dtype=torch.complex64,
                                                                                      device=d), (16, 16))
    assert torch.count_nonzero(z) == 0


def test_out_of_range_coordinates_wrap():
    rng = np.random.default_rng(42)
    x = rng.uniform(np.pi, 3 * np.pi, 50).astype(np.float32)
    c = rand_c(rng, 50)
    a = nb.nufft1d1(to_dev(x), to_dev(c), 32).cpu().numpy()
    b = nb.nufft1d1(to_dev(np.mod(x + np.pi, 2 * np.pi) - np.pi), to_dev(c), 32).cpu().numpy()
    assert np.allclose(a, b, rtol=1e-4, atol=1e-4)


def test_empty_points():
    d = dev()
    f = nb.nufft2d1(torch.zeros(0, device=d), torch.zeros(0, device=d), torch.zeros(0, dtype=torch.complex64, device=d),
                    (8, 8))
    assert f.shape == (8, 8) and torch.count_nonzero(f) == 0
    c = nb.nufft2d2(torch.zeros(0, device=d), torch.zeros(0, device=d), torch.ones((8, 8), dtype=torch.complex64,
                                                                                   device=d))
    assert c.shape == (0,)


# -- odd sizes, odd fine grids, batches, isign 0 ---------------------------------------
@pytest.mark.parametrize("dim,n_modes", [(1, (63,)), (2, (31, 17)), (3, (9, 12, 7)), (2, (100, 50))])
@pytest.mark.parametrize("uf", [2.0, 1.25])
def test_odd_modes_and_grids(dim, n_modes, uf):
    rng = np.random.default_rng(500 + dim)
    M = 3000
    eps = 1e-9
    X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
    c = rand_c(rng, (2, M), np.complex128)
    f = rand_c(rng, (2,) + tuple(reversed(n_modes)), np.complex128)
    t1 = {1: nb.nufft1d1, 2: nb.nufft2d1, 3: nb.nufft3d1}[dim]
    t2 = {1: nb.nufft1d2, 2: nb.nufft2d2, 3: nb.nufft3d2}[dim]
    nm = n_modes[0] if dim == 1 else n_modes
    Xd = [to_dev(x) for x in X]
    a = t1(*Xd, to_dev(c), nm, eps=eps, upsampfac=uf).cpu().numpy()
    b = t2(*Xd, to_dev(f), eps=eps, upsampfac=uf).cpu().numpy()
    assert a.shape == (2,) + tuple(reversed(n_modes)) and b.shape == (2, M)
    assert rel_l2(a, O.nufft_type1(X, c, n_modes, eps=eps, upsampfac=uf)) <= 2 * eps
    assert rel_l2(b, O.nufft_type2(X, f, eps=eps, upsampfac=uf)) <= 2 * eps
    if uf == 2.0:
        assert rel_l2(a[0], O.direct_type1(X, c[0], n_modes)) < 10 * eps


def test_isign_zero_follows_reference_fft_choice():
    """isign = 0: type 1 takes the forward FFT (nufft1.py:81), type 2 the inverse (nufft2.py:81)."""
    rng = np.random.default_rng(77)
    X = [rng.uniform(-np.pi, np.pi, 500) for _ in range(2)]
    c = rand_c(rng, 500, np.complex128)
    f = rand_c(rng, (12, 10), np.complex128)
    Xd = [to_dev(x) for x in X]
    a = nb.nufft2d1(*Xd, to_dev(c), (10, 12), eps=1e-9, isign=0).cpu().numpy()
    b = nb.nufft2d2(*Xd, to_dev(f), eps=1e-9, isign=0).cpu().numpy()
    assert rel_l2(a, O.nufft_type1(X, c, (10, 12), eps=1e-9, isign=0)) <= 2e-9
    assert rel_l2(b, O.nufft_type2(X, f, eps=1e-9, isign=0)) <= 2e-9


def test_noncontiguous_and_mixed_dtype_inputs():
    rng = np.random.default_rng(78)
    xy = to_dev(rng.uniform(-np.pi, np.pi, (1000, 2)).astype(np.float32))
    c = to_dev(rand_c(rng, 1000))
    f = nb.nufft2d1(xy[:, 0], xy[:, 1], c, (16, 16)).cpu().numpy()  # strided coordinates
    X = [xy[:, 0].cpu().numpy(), xy[:, 1].cpu().numpy()]
    assert rel_l2(f, O.nufft_type1(X, c.cpu().numpy(), (16, 16))) <= 2e-6
    # float64 coordinates with complex64 strengths compute in the strengths' precision
    g = nb.nufft2d1(xy[:, 0].double(), xy[:, 1].double(), c, (16, 16))
    assert g.dtype == torch.complex64
    assert rel_l2(g.cpu().numpy(), f) < 1e-6
