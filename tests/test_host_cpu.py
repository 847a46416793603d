"""CPU: the C-ABI library loads and exports include/nfx.h; host-side logic.

No compute call is made here (there is no GPU): only option resolution,
workspace sizing and argument validation, which return before touching CUDA.
"""

import ctypes
from ctypes import byref, c_size_t

import numpy as np
import pytest

import nufftax_b200 as nb
from nufftax_b200 import _lib
from nufftax_b200.kernel import deconv_factors
from oracle import nufft_oracle as O


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    names = _lib.header_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert lib.nfx_version() >= 10000


def test_signatures_cover_header():
    assert set(_lib.header_symbols()) == set(_lib._SIGNATURES)


def _opts(dim=2, nf=(1024, 1024), ns=8, precision=0):
    o = _lib.NfxOpts()
    o.precision = precision
    o.dim = dim
    o.nf = _lib.int3(nf)
    o.nspread = ns
    o.beta = 18.6
    o.kc = 4.0 / max(ns, 1) ** 2
    return o


def test_default_tiles_and_workspace():
    lib = _lib.load()
    o = _opts()
    assert lib.nfx_default_tiles(byref(o)) == 0
    # max_subproblem = 0 stays "auto": the sort layout picks it from M
    assert list(o.tile)[:2] == [32, 32] and o.max_subproblem == 0
    b = c_size_t(0)
    assert lib.nfx_sort_workspace_bytes(byref(o), 4_000_000, byref(b)) == 0
    assert 8 * 4_000_000 < b.value < 64 * 4_000_000


@pytest.mark.parametrize("M,expected", [(500_000, 1024), (3_000_000, 1024), (4_000_000, 2048),
                                        (20_000_000, 4096)])
def test_auto_subproblem_size(M, expected):
    """2D default: 1024, doubled (up to 4096) while M / (2 * size) >= 1480; the
    workspace of max_subproblem = 0 equals that of the explicit size."""
    lib = _lib.load()
    auto, explicit = _opts(), _opts()
    assert lib.nfx_default_tiles(byref(auto)) == 0
    assert lib.nfx_default_tiles(byref(explicit)) == 0
    explicit.max_subproblem = expected
    ba, be = c_size_t(0), c_size_t(0)
    assert lib.nfx_sort_workspace_bytes(byref(auto), M, byref(ba)) == 0
    assert lib.nfx_sort_workspace_bytes(byref(explicit), M, byref(be)) == 0
    assert ba.value == be.value
    o3 = _opts(3, (256, 256, 256))
    assert lib.nfx_default_tiles(byref(o3)) == 0
    assert all(t > 0 for t in o3.tile)


@pytest.mark.parametrize("ns,code", [(3, _lib.NFX_ERR_UNSUPPORTED), (18, _lib.NFX_ERR_UNSUPPORTED),
                                     (0, _lib.NFX_ERR_UNSUPPORTED)])
def test_invalid_nspread_rejected(ns, code):
    lib = _lib.load()
    o = _opts(ns=ns)
    assert lib.nfx_default_tiles(byref(o)) == code
    assert b"nspread" in lib.nfx_last_error()


def test_invalid_arguments_rejected_without_gpu():
    lib = _lib.load()
    o = _opts()
    o.dim = 4
    assert lib.nfx_default_tiles(byref(o)) == _lib.NFX_ERR_INVALID
    o = _opts()
    # workspace too small is reported before any device work
    assert lib.nfx_sort_points(byref(o), ctypes.c_void_p(8), ctypes.c_void_p(8), None, 10, ctypes.c_void_p(8), 4,
                               None) == _lib.NFX_ERR_WORKSPACE
    # missing coordinate pointer
    assert lib.nfx_spread(byref(o), ctypes.c_void_p(8), None, None, 10, ctypes.c_void_p(8), 1, ctypes.c_void_p(8),
                          ctypes.c_void_p(8), 1 << 30, None) == _lib.NFX_ERR_INVALID
    # FFT with a bad sign / deconvolution with more modes than grid
    assert lib.nfx_fft(0, 2, _lib.int3((8, 8)), 1, ctypes.c_void_p(8), 0, None) == _lib.NFX_ERR_INVALID
    assert lib.nfx_deconv_pad(0, 1, _lib.int3((8,)), _lib.int3((9,)), ctypes.c_void_p(8), None, None,
                              ctypes.c_void_p(8), ctypes.c_void_p(8), 1, None) == _lib.NFX_ERR_INVALID
    # one-call transforms without options; FFT entries with a bad sign / no size pointer
    assert lib.nfx_nufft1(None, _lib.int3((8, 8)), None, None, None, 0, None, 1, 1, None, None, None, None, None,
                          None, 0, None) == _lib.NFX_ERR_INVALID
    assert lib.nfx_nufft2(None, _lib.int3((8, 8)), None, None, None, 0, None, 1, -1, None, None, None, None, None,
                          None, 0, None) == _lib.NFX_ERR_INVALID
    assert lib.nfx_fft_ws(0, 2, _lib.int3((8, 8)), 1, ctypes.c_void_p(8), 2, None, 0, None) == _lib.NFX_ERR_INVALID
    assert lib.nfx_fft_ws(0, 2, _lib.int3((8, 8)), 1, None, 1, None, 0, None) == _lib.NFX_ERR_INVALID
    assert lib.nfx_fft_work_bytes(0, 2, _lib.int3((8, 8)), 1, None) == _lib.NFX_ERR_INVALID
    with pytest.raises(ValueError):
        _lib.check(_lib.NFX_ERR_INVALID, "probe")


@pytest.mark.parametrize("eps", [1e-2, 1e-3, 1e-5, 1e-6, 1e-9, 1e-12, 1e-15])
@pytest.mark.parametrize("uf", [2.0, 1.25])
def test_kernel_params_match_oracle(eps, uf):
    a = nb.compute_kernel_params(eps, uf)
    b = O.compute_kernel_params(eps, uf)
    assert tuple(a) == tuple(b)


def test_grid_helpers_match_oracle():
    for n in [1, 7, 64, 128, 384, 512, 1000, 8192]:
        for uf in (2.0, 1.25):
            assert nb.compute_grid_size(n, uf, 8) == O.compute_grid_size(n, uf, 8)
    assert nb.compute_type3_grid_size(np.pi, 300.0, eps=1e-6) == 1250
    x = np.linspace(-np.pi, np.pi, 11)
    s = np.linspace(-300, 300, 7)
    assert nb.compute_type3_grid_size(x, s) == 1250
    assert nb.compute_type3_grid_sizes_2d(np.pi, np.pi, 300, 300) == (1250, 1250)
    assert nb.compute_type3_grid_sizes_3d(1.0, 2.0, 3.0, 10, 20, 30) == tuple(
        O.type3_grid_size(e, s, 1e-6) for e, s in ((1.0, 10), (2.0, 20), (3.0, 30)))


@pytest.mark.parametrize("nf,n", [(256, 128), (1024, 512), (20, 7), (16, 16)])
def test_deconv_factors_match_oracle(nf, n):
    kp = nb.compute_kernel_params(1e-6)
    ph = O.kernel_fourier_series(nf, kp.nspread, kp.beta, kp.c)
    assert np.allclose(deconv_factors(nf, n, kp), O.deconv_factors_1d(ph, n), rtol=1e-14)


def test_upsampfac_split():
    from nufftax_b200.transforms import _split_upsampfac

    assert _split_upsampfac(2.0) == (2.0, 2.0)
    assert _split_upsampfac((2.0, 1.25)) == (2.0, 1.25)


def test_product_does_not_import_oracle():
    import pathlib

    pkg = pathlib.Path(nb.__file__).parent
    for f in pkg.rglob("*.py"):
        assert "oracle" not in f.read_text().replace("oracle is", ""), f


@pytest.mark.parametrize("eps", [1e-6, 1e-9, 1e-12])
def test_es_polynomial_matches_exp_sqrt(eps):
    """The float kernels' polynomial ES weights (nfx_es_poly, host-side fit) stay
    within about two float ulps (2.6e-7 relative, +3e-8) of
    exp(beta (sqrt(1 - c z^2) - 1)), by Horner's rule and by the even / odd
    split the kernels use for whole footprints; weight ns - 1 - q is weight q
    at -v."""
    lib = _lib.load()
    kp = nb.compute_kernel_params(eps)
    co = (ctypes.c_float * 256)()
    deg = ctypes.c_int()
    err = ctypes.c_double()
    assert lib.nfx_es_poly(kp.nspread, kp.beta, kp.c, co, byref(deg), byref(err)) == 0
    assert deg.value > 0
    a = np.frombuffer(co, dtype=np.float32).reshape(16, 16)
    v = np.linspace(-1, 1, 1001).astype(np.float32)
    for q in range(kp.nspread):
        h = np.full_like(v, a[q, deg.value])
        for d in range(deg.value - 1, -1, -1):
            h = (h.astype(np.float64) * v + a[q, d]).astype(np.float32)
        z = q - (v.astype(np.float64) + kp.nspread - 1) / 2
        ref = O.es_kernel(z, kp.beta, kp.c)
        assert np.all(np.abs(h - ref) <= 3e-8 + 2.6e-7 * np.abs(ref) + 1e-7)
    ns = kp.nspread
    sign = np.array([(-1) ** d for d in range(16)], dtype=np.float32)
    for q in range(ns // 2):
        assert np.array_equal(a[ns - 1 - q], a[q] * sign)
        u = (v.astype(np.float64) * v).astype(np.float32)
        e, o = np.full_like(v, a[q, 6]), np.full_like(v, a[q, 7])
        for d in (4, 2, 0):
            e = (e.astype(np.float64) * u + a[q, d]).astype(np.float32)
            o = (o.astype(np.float64) * u + a[q, d + 1]).astype(np.float32)
        for s_, qq in ((1.0, q), (-1.0, ns - 1 - q)):
            w = (np.float64(s_) * v * o + e).astype(np.float32)
            ref = O.es_kernel(qq - (v.astype(np.float64) + ns - 1) / 2, kp.beta, kp.c)
            assert np.all(np.abs(w - ref) <= 3e-8 + 2.6e-7 * np.abs(ref) + 1e-7)


def test_es_polynomial_refused_for_narrow_kernel():
    lib = _lib.load()
    kp = nb.compute_kernel_params(1e-3)  # ns = 4: too much edge mass for a float-accurate fit
    deg = ctypes.c_int()
    assert lib.nfx_es_poly(kp.nspread, kp.beta, kp.c, None, byref(deg), None) == 0
    assert deg.value == 0


def test_make_opts_cache_returns_private_copies():
    """make_opts caches the filled struct per key but hands out copies: changing
    one caller's options leaves the cache and other callers untouched."""
    from nufftax_b200._plan import make_opts

    kp = nb.compute_kernel_params(1e-6)
    a = make_opts(0, (1024, 1024), kp, True)
    b = make_opts(0, (1024, 1024), kp, True)
    assert a is not b and bytes(a) == bytes(b)
    a.max_subproblem = 77
    a.tile[0] = 5
    c = make_opts(0, (1024, 1024), kp, True)
    assert bytes(c) == bytes(b) and c.max_subproblem == 0 and c.tile[0] == 32
    d = make_opts(0, (1024, 1024), kp, True, tile=(16, 16))
    assert list(d.tile)[:2] == [16, 16]
    bad = nb.compute_kernel_params(1e-6)._replace(nspread=18)
    for _ in range(2):  # a failed fill is not cached
        with pytest.raises(NotImplementedError):
            make_opts(0, (1024, 1024), bad, True)


def test_profiling_span_is_inert_without_recorder():
    """Outside profiling.record() a span touches no CUDA state (this runs without a GPU)."""
    from nufftax_b200 import profiling

    with profiling.span("nfx_spread_sorted", None) as s:
        assert s.rec is None
    assert profiling.LAUNCHES["nfx_sort_points"] >= 1
    # a recorder limited to some calls leaves the others inert, and a lazily
    # given launch count is never evaluated for them
    with profiling.record(only=["nfx_spread_sorted"]) as rec:
        with profiling.span("nfx_interp_sorted", None, lambda: 1 / 0) as s:
            assert s.rec is None
    assert rec.events == []


def test_autotune_cache_round_trip(tmp_path, monkeypatch):
    """The tuner's JSON cache (NUFFTAX_B200_TUNE_CACHE) loads what it saved and
    ignores a malformed file."""
    from nufftax_b200 import autotune

    path = tmp_path / "tune.json"
    monkeypatch.setenv("NUFFTAX_B200_TUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "_cache", {})
    monkeypatch.setattr(autotune, "_loaded", True)
    autotune._cache["d2-uf2-ns8-f32-rho2-clu"] = ((32, 32), 2048, (3, 2))
    autotune._save()
    monkeypatch.setattr(autotune, "_cache", {})
    monkeypatch.setattr(autotune, "_loaded", False)
    assert autotune.cached() == {"d2-uf2-ns8-f32-rho2-clu": ((32, 32), 2048, (3, 2))}
    path.write_text("{not json")
    monkeypatch.setattr(autotune, "_cache", {})
    monkeypatch.setattr(autotune, "_loaded", False)
    assert autotune.cached() == {}


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-12])
def test_deconv_factors_positive_symmetric_growing(eps):
    """Properties the reference's kernel tests check on phi-hat
    (nufftax tests/test_kernel.py): the Fourier series is positive and decays
    away from k = 0, so the per-mode factors 1 / phi-hat are positive, symmetric
    in k and grow with |k|."""
    kp = nb.compute_kernel_params(eps)
    n = 64
    nf = nb.compute_grid_size(n, 2.0, kp.nspread)
    fac = np.abs(deconv_factors(nf, n, kp))  # CMCL order k = -n/2 .. n/2 - 1, sign (-1)^k
    assert np.all(fac > 0)
    k = np.arange(-n // 2, n // 2)
    mag = {int(kk): f for kk, f in zip(k, fac)}
    for kk in range(1, n // 2):
        assert np.isclose(mag[kk], mag[-kk], rtol=1e-12)
        assert mag[kk] >= mag[kk - 1]


def test_host_only_sizes_and_limits():
    """Entry points that size buffers or set limits answer without a GPU: the
    no-alloc scratch (64 MiB), type-3 parameter / scratch sizes, the batched
    deconvolution table (growing with the problem count), the FFT plan-cache limit
    (at least one plan) and the SM count (a default without a device)."""
    lib = _lib.load()
    assert lib.nfx_noalloc_scratch_bytes() == 64 << 20
    assert lib.nfx_t3_params_bytes() > 0
    assert lib.nfx_t3_scratch_bytes(0, 1000, 2000) > 0 and lib.nfx_t3_scratch_bytes(1, 1000, 2000) > 0
    sizes = [lib.nfx_batch_deconv_table_bytes(0, n) for n in (1, 2, 8, 64)]
    assert sizes[0] > 0 and all(a <= b for a, b in zip(sizes, sizes[1:])) and sizes[-1] > sizes[0]
    assert lib.nfx_fft_cache_limit(0) == _lib.NFX_ERR_INVALID
    assert lib.nfx_fft_cache_limit(1024) == 0
    assert lib.nfx_num_sms() >= 1


def test_batch_info_host_side():
    """nfx_batch_info_get sizes the device table, the shared memory and the
    work-queue bound of a batched launch from the problem descriptors alone."""
    lib = _lib.load()
    kp = nb.compute_kernel_params(1e-6)
    common = _lib.NfxOpts()
    common.precision, common.dim, common.nspread, common.prenorm = 0, 2, int(kp.nspread), 1
    common.beta, common.kc = float(kp.beta), float(kp.c)

    def info_for(specs):
        probs = (_lib.NfxBatchProblem * len(specs))()
        for i, (M, nf) in enumerate(specs):
            probs[i].M = M
            probs[i].nf = _lib.int3(nf)
        info = _lib.NfxBatchInfo()
        assert lib.nfx_batch_info_get(byref(common), 1, probs, len(specs), byref(info)) == 0, lib.nfx_last_error()
        return info

    a = info_for([(1000, (64, 64))])
    b = info_for([(1000, (64, 64)), (50_000, (256, 192))])
    assert a.table_bytes > 0 and a.smem_bytes > 0 and a.max_subs >= 1
    assert b.table_bytes > a.table_bytes and b.max_subs > a.max_subs


def test_sort_kernel_count():
    """The library's count of the kernels one sort launches: 2D 1024^2 with 32^2
    tiles is two 10-bit passes (keys, 2 x (scan, scatter), count, subproblems;
    the coordinates ride through the passes and the last pass writes the bin
    starts); a 3D 320^3 sort three 8-bit passes plus bin bounds; type-3 and
    double points add the coordinate gather; an empty sort runs bin bounds and
    subproblems only."""
    from nufftax_b200._plan import make_opts, sort_launches

    kp = nb.compute_kernel_params(1e-6)
    o2 = make_opts(_lib.NFX_F32, (1024, 1024), kp, True)
    assert sort_launches(o2, 4_000_000) == 7
    assert sort_launches(o2, 4_000_000, type3=True) == 8
    assert sort_launches(make_opts(_lib.NFX_F64, (1024, 1024), kp, True), 4_000_000) == 8
    o3 = make_opts(_lib.NFX_F32, (320, 320, 320), kp, True)
    assert sort_launches(o3, 10_000) == 11
    assert sort_launches(o2, 0) == 2
