"""CPU: pin the oracle to the reference's own test oracles and known answers.

The reference cannot run here (no JAX), so these tests check the NumPy
restatement against what the reference's tests check it against: FP64 direct
sums (tests/conftest.py:154-198, tests/test_nufft3.py:26-72), known answers
(tests/test_edge_cases.py), the spread/interp adjoint identity
(tests/test_spread.py:300-347), the kernel parameter formulas
(nufftax/core/kernel.py:165-206) and the committed golden fixtures.
"""

import numpy as np
import pytest

from oracle import nufft_oracle as O
from tests.conftest import GOLDEN, rel_l2


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


# -- kernel parameters / grid sizes --------------------------------------------------------
@pytest.mark.parametrize("eps,ns,beta", [(1e-6, 8, 18.6389), (1e-5, 6, 13.8551), (1e-12, 14, 32.8668),
                                         (1e-3, 4, 8.99615), (1e-9, 10, 23.3938)])
def test_kernel_params_table(eps, ns, beta):
    kp = O.compute_kernel_params(eps)
    assert kp.nspread == ns
    assert kp.beta == pytest.approx(beta, rel=1e-5)
    assert kp.c == pytest.approx(4.0 / ns**2)


def test_kernel_params_clamps():
    assert O.compute_kernel_params(1.0).nspread == 2
    assert O.compute_kernel_params(1e-20).nspread == 16
    assert O.compute_kernel_params(1e-6, upsampfac=1.25).beta < O.compute_kernel_params(1e-6).beta


@pytest.mark.parametrize("n,nf", [(128, 256), (512, 1024), (8192, 16384), (384, 768), (160, 320), (1, 16), (7, 16)])
def test_grid_sizes(n, nf):
    assert O.compute_grid_size(n, 2.0, 8) == nf


def test_smooth_numbers():
    for n in range(1, 500):
        m = O.next_smooth_int(n)
        assert m >= n
        v = m
        for p in (2, 3, 5):
            while v % p == 0:
                v //= p
        assert v == 1
    assert O.next_smooth_even(7) == 8 and O.next_smooth_even(1) == 2
    # type-3 grid at X = pi, S = 300, eps = 1e-6 (nufft3.py:103-104): nf = 1250
    assert O.type3_grid_size(np.pi, 300.0, 1e-6) == 1250


def test_es_kernel_properties():
    kp = O.compute_kernel_params(1e-6)
    z = np.linspace(-4, 4, 101)
    phi = O.es_kernel(z, kp.beta, kp.c)
    assert phi[50] == pytest.approx(1.0)
    assert np.allclose(phi, phi[::-1])
    assert np.all(np.diff(phi[50:]) <= 0)
    assert O.es_kernel(np.array([4.5]), kp.beta, kp.c)[0] == 0.0
    ph = O.kernel_fourier_series(256, kp.nspread, kp.beta, kp.c)
    assert np.all(ph > 0)


# -- folding -----------------------------------------------------------------------------
def test_premod_matches_jnp_mod_semantics():
    x = np.array([np.pi, -np.pi, 0.0, 3.5, -3.5, 7.0, -7.0, 1e-8, -1e-8], dtype=np.float32)
    r = O.premod(x)
    assert r.dtype == np.float32
    assert np.all(r >= np.float32(-np.pi)) and np.all(r <= np.float32(np.pi))
    # the float32 sum x + pi then fmod: x = -pi lands exactly on -pi
    assert r[1] == np.float32(-np.pi)


def test_fold_rescale_range_and_dtype():
    x = np.random.default_rng(0).uniform(-10, 10, 10000).astype(np.float32)
    xs = O.fold_rescale(x, 256)
    assert xs.dtype == np.float32
    assert np.all(xs >= 0) and np.all(xs <= 256)


# -- bin sort fixtures --------------------------------------------------------------------
@pytest.mark.parametrize("name", ["sort_1d", "sort_2d", "sort_3d"])
def test_sort_fixture_reproduces(name):
    d = load(name)
    dim = len(d["nf"])
    X = [d[f"x{i}"] for i in range(dim)]
    nbins = int(np.prod([-(-n // t) for n, t in zip(d["nf"], d["tile"])]))
    ncell = int(np.prod(d["tile"]))
    for p in (0, 1):
        keys, cells = O.bin_keys(X, d["nf"], int(d["ns"]), d["tile"], bool(p))
        assert np.array_equal(keys, d[f"keys_p{p}"])
        assert np.array_equal(cells, d[f"cells_p{p}"])
        perm, bs = O.bin_sort(keys, cells, nbins, ncell)
        assert np.array_equal(perm, d[f"perm_p{p}"])
        assert np.array_equal(bs, d[f"bin_start_p{p}"])
        # ordered by (bin, cell); stable: equal keys keep the original order
        fine = keys.astype(np.int64)[perm] * ncell + cells[perm]
        assert np.all(np.diff(fine) >= 0)
        same = np.diff(fine) == 0
        assert np.all(np.diff(perm)[same] > 0)


# -- transforms against direct sums ------------------------------------------------------
@pytest.mark.parametrize("name", ["t1_1d", "t1_2d", "t1_3d"])
def test_type1_oracle_vs_direct(name):
    d = load(name)
    dim = len(d["n_modes"])
    X = [d[f"x{i}"] for i in range(dim)]
    for e in d["eps"]:
        f = O.nufft_type1(X, d["c"], tuple(d["n_modes"]), eps=float(e), isign=int(d["isign"]))
        assert np.allclose(f, d[f"oracle_{e:g}"], rtol=0, atol=1e-12 * np.abs(f).max())
        # reference tests accept 10*eps against an exact transform (test_nufft1.py:118)
        assert rel_l2(f, d["direct"]) < 10 * e


@pytest.mark.parametrize("name", ["t2_1d", "t2_2d", "t2_3d"])
def test_type2_oracle_vs_direct(name):
    d = load(name)
    dim = d["f"].ndim
    X = [d[f"x{i}"] for i in range(dim)]
    for e in d["eps"]:
        c = O.nufft_type2(X, d["f"], eps=float(e), isign=int(d["isign"]))
        assert np.allclose(c, d[f"oracle_{e:g}"], rtol=0, atol=1e-12 * np.abs(c).max())
        assert rel_l2(c, d["direct"]) < 10 * e


@pytest.mark.parametrize("name", ["t3_1d", "t3_2d", "t3_3d"])
def test_type3_oracle_vs_direct(name):
    d = load(name)
    dim = len(d["nf"])
    src = [d[f"x{i}"] for i in range(dim)]
    tgt = [d[f"s{i}"] for i in range(dim)]
    f = O.nufft_type3(src, d["c"], tgt, tuple(d["nf"]), eps=1e-6)
    assert np.allclose(f, d["oracle_1e-06"], rtol=0, atol=1e-12 * np.abs(f).max())
    # tests/test_nufft3.py:48 asserts < 1e-4 against the direct sum at eps = 1e-6
    assert rel_l2(f, d["direct"]) < 1e-4


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-9, 1e-12])
def test_type1_accuracy_contract(eps):
    """rel l2 against the direct sum stays within 2 eps at upsampfac 2."""
    rng = np.random.default_rng(3)
    x = rng.uniform(-np.pi, np.pi, 3000)
    c = rng.standard_normal(3000) + 1j * rng.standard_normal(3000)
    f = O.nufft_type1([x], c, (256,), eps=eps)
    assert rel_l2(f, O.direct_type1([x], c, (256,))) < 2 * eps


# -- known answers (tests/test_edge_cases.py) --------------------------------------------
def test_known_single_point():
    f = O.nufft_type1([np.array([0.5])], np.array([1 + 1j]), (16,))
    k = np.arange(-8, 8)
    assert np.allclose(f, (1 + 1j) * np.exp(1j * k * 0.5), rtol=1e-5)


def test_known_points_at_origin_and_pi():
    f = O.nufft_type1([np.zeros(10)], np.ones(10, complex), (32,))
    assert np.allclose(f, 10, rtol=1e-5)
    f = O.nufft_type1([np.full(10, np.pi)], np.ones(10, complex), (32,))
    k = np.arange(-16, 16)
    assert np.allclose(f, 10 * np.exp(1j * k * np.pi), rtol=1e-5)


def test_known_regular_grid():
    N = 32
    x = np.linspace(-np.pi, np.pi, N, endpoint=False)
    f = O.nufft_type1([x], np.ones(N, complex), (N,))
    assert abs(abs(f[N // 2]) - N) < 1e-5 * N
    assert np.max(np.abs(np.delete(f, N // 2))) < 1e-4


def test_known_wrap_and_zero():
    rng = np.random.default_rng(42)
    x = rng.uniform(np.pi, 3 * np.pi, 50)
    c = rng.standard_normal(50) + 1j * rng.standard_normal(50)
    a = O.nufft_type1([x], c, (32,))
    b = O.nufft_type1([np.mod(x + np.pi, 2 * np.pi) - np.pi], c, (32,))
    assert np.allclose(a, b, rtol=1e-5)
    z = O.nufft_type1([x], np.zeros(50, complex), (32,))
    assert np.all(z == 0)


def test_adjoint_identity():
    """<spread c, fw> = <c, interp fw> to 1e-10 (tests/test_spread.py:300-347)."""
    rng = np.random.default_rng(42)
    kp = O.compute_kernel_params(1e-6)
    for dim, nf in ((1, (64,)), (2, (32, 24)), (3, (16, 12, 20))):
        X = [rng.uniform(-np.pi, np.pi, 50) for _ in range(dim)]
        c = rng.standard_normal(50) + 1j * rng.standard_normal(50)
        fw = rng.standard_normal(tuple(reversed(nf))) + 1j * rng.standard_normal(tuple(reversed(nf)))
        lhs = np.vdot(O.spread(X, c, nf, kp), fw)
        rhs = np.vdot(c, O.interp(X, fw, kp))
        assert abs(lhs - rhs) / abs(lhs) < 1e-10


def test_type1_type2_adjoint():
    rng = np.random.default_rng(5)
    x, y = rng.uniform(-np.pi, np.pi, (2, 300))
    c = rng.standard_normal(300) + 1j * rng.standard_normal(300)
    f = rng.standard_normal((12, 16)) + 1j * rng.standard_normal((12, 16))
    a = np.vdot(f, O.nufft_type1([x, y], c, (16, 12), isign=1, eps=1e-9))
    b = np.vdot(O.nufft_type2([x, y], f, isign=-1, eps=1e-9), c)
    assert abs(a - b) / abs(a) < 1e-8


@pytest.mark.parametrize("eps,bound", [(1e-3, 2e-2), (1e-6, 1e-4), (1e-9, 1e-5)])
def test_upsampfac_125_works_but_coarse(eps, bound):
    """nufftax tests/test_upsampfac.py: upsampfac 1.25 runs with the same kernel
    width and is coarser than 2.0 but still converges with eps (types 1 and 2
    against the direct sums)."""
    rng = np.random.default_rng(3)
    x = rng.uniform(-np.pi, np.pi, 3000)
    c = rng.standard_normal(3000) + 1j * rng.standard_normal(3000)
    fm = rng.standard_normal(256) + 1j * rng.standard_normal(256)
    d1 = O.direct_type1([x], c, (256,))
    d2 = O.direct_type2([x], fm, O.flat_mode_list((256,)))
    e1 = {uf: rel_l2(O.nufft_type1([x], c, (256,), eps=eps, upsampfac=uf), d1) for uf in (2.0, 1.25)}
    e2 = {uf: rel_l2(O.nufft_type2([x], fm, eps=eps, upsampfac=uf), d2) for uf in (2.0, 1.25)}
    assert O.compute_kernel_params(eps, 1.25).nspread == O.compute_kernel_params(eps, 2.0).nspread
    for e in (e1, e2):
        assert e[2.0] < 2 * eps and e[1.25] < bound and e[1.25] > e[2.0]
