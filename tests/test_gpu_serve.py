"""GPU: the continuous-batching server returns, for every request of a mixed
stream served concurrently, the same result as the request alone through the
public API (relative l2 <= 2 eps, eps = 1e-6), and honours its memory budget."""

import numpy as np
import pytest
import torch

import nufftax_b200 as nb
from nufftax_b200 import profiling
from nufftax_b200.serve import NufftServer, Request
from tests.conftest import cuda_device, rel_l2

pytestmark = pytest.mark.gpu


def _mix(rng, dev, n=30):
    reqs = []
    for i in range(n):
        kind = [1, 2, 3][i % 3]
        dim = 3 if (i % 5 == 1 and kind != 3) else 2
        M = int(rng.integers(500, 40000))
        X = [torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev) for _ in range(dim)]
        if kind == 3:
            T = [torch.from_numpy(rng.uniform(-40, 40, M).astype(np.float32)).to(dev) for _ in range(dim)]
            nm = nb.compute_type3_grid_sizes_2d(np.pi, np.pi, 40.0, 40.0, eps=1e-6)
            c = torch.from_numpy((rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)).to(dev)
            reqs.append(Request(kind=3, dim=2, n_modes=nm, M=M, K=M, coords=X, strengths=c, targets=T))
            continue
        nm = tuple(int(rng.choice([16, 24, 32, 48])) for _ in range(dim))
        if kind == 1:
            c = torch.from_numpy((rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)).to(dev)
        else:
            shape = tuple(reversed(nm))
            c = torch.from_numpy((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(
                np.complex64)).to(dev)
        reqs.append(Request(kind=kind, dim=dim, n_modes=nm, M=M, coords=X, strengths=c,
                            points_id=("pts", i // 6) if i % 6 == 0 else None))
    return reqs


def _alone(r):
    if r.kind == 1:
        return {2: nb.nufft2d1, 3: nb.nufft3d1}[r.dim](*r.coords, r.strengths, r.n_modes)
    if r.kind == 2:
        return {2: nb.nufft2d2, 3: nb.nufft3d2}[r.dim](*r.coords, r.strengths)
    return nb.nufft2d3(*r.coords, r.strengths, *r.targets, r.n_modes)


def test_mix_equals_alone():
    dev = cuda_device()
    rng = np.random.default_rng(8)
    reqs = _mix(rng, dev)
    server = NufftServer(dev, slots=6, hbm_budget=2e9)
    done = server.serve(reqs, list(np.linspace(0, 0.02, len(reqs))))
    assert len(done) == len(reqs)
    torch.cuda.synchronize()
    for r in reqs:
        ref = _alone(r)
        assert rel_l2(r.result.cpu().numpy(), ref.cpu().numpy()) <= 2e-6
    st = server.stats(done)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert server.in_use == 0


def test_budget_serialises_large_requests():
    dev = cuda_device()
    rng = np.random.default_rng(9)
    reqs = _mix(rng, dev, n=12)
    budget = max(r_bytes for r_bytes in [__import__("nufftax_b200.serve").serve.estimate_bytes(r) for r in reqs])
    server = NufftServer(dev, slots=8, hbm_budget=budget)
    peak = 0
    orig = server._admit

    def watched():
        nonlocal peak
        orig()
        peak = max(peak, server.in_use)

    server._admit = watched
    done = server.serve(reqs)
    assert len(done) == 12 and peak <= budget
    for r in reqs:
        assert rel_l2(r.result.cpu().numpy(), _alone(r).cpu().numpy()) <= 2e-6


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_one_call_entry_points_match_api(dim, dtype):
    """nfx_nufft1 / nfx_nufft2 (sort + spread/interp + FFT + deconvolution in one
    library call, two transforms) equal the public API transform by transform."""
    from ctypes import byref, c_size_t, c_void_p

    from nufftax_b200 import _lib
    from nufftax_b200._plan import _facs, make_opts, ptr
    from nufftax_b200.grid import compute_grid_size
    from nufftax_b200.kernel import compute_kernel_params

    dev = cuda_device()
    rng = np.random.default_rng(20 + dim)
    eps = 1e-6 if dtype == torch.complex64 else 1e-9
    prec = _lib.NFX_F32 if dtype == torch.complex64 else _lib.NFX_F64
    rdt = torch.float32 if dtype == torch.complex64 else torch.float64
    M, nt = 3000, 2
    nm = (40, 24, 16)[:dim]
    X = [torch.from_numpy(rng.uniform(-np.pi, np.pi, M)).to(dev, rdt) for _ in range(dim)]
    c = torch.from_numpy(rng.standard_normal((nt, M)) + 1j * rng.standard_normal((nt, M))).to(dev, dtype)
    f = torch.from_numpy(rng.standard_normal((nt,) + nm[::-1]) + 1j * rng.standard_normal((nt,) + nm[::-1])).to(
        dev, dtype)
    kp = compute_kernel_params(eps)
    nf = tuple(compute_grid_size(n, 2.0, kp.nspread) for n in nm)
    o = make_opts(prec, nf, kp, prenorm=True)
    lib = _lib.load()
    nb_ = c_size_t(0)
    assert lib.nfx_sort_workspace_bytes(byref(o), M, byref(nb_)) == 0
    ws = torch.empty(nb_.value, dtype=torch.uint8, device=dev)
    fw = torch.empty((nt,) + nf[::-1], dtype=dtype, device=dev)
    facs = [ptr(t) for t in _facs(nf, nm, kp, prec, dev)]
    xyz = [ptr(x) for x in X] + [None] * (3 - dim)
    st = c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    F = torch.empty((nt,) + nm[::-1], dtype=dtype, device=dev)
    C = torch.empty((nt, M), dtype=dtype, device=dev)
    # type 1 with isign +1 runs the FFT with sign +1; type 2 with isign -1 with sign -1
    assert lib.nfx_nufft1(byref(o), _lib.int3(nm), *xyz, M, ptr(c), nt, 1, *facs, ptr(fw), ptr(F), ptr(ws),
                          ws.numel(), st) == 0, lib.nfx_last_error()
    assert lib.nfx_nufft2(byref(o), _lib.int3(nm), *xyz, M, ptr(f), nt, -1, *facs, ptr(fw), ptr(C), ptr(ws),
                          ws.numel(), st) == 0, lib.nfx_last_error()
    t1 = {1: nb.nufft1d1, 2: nb.nufft2d1, 3: nb.nufft3d1}[dim]
    t2 = {1: nb.nufft1d2, 2: nb.nufft2d2, 3: nb.nufft3d2}[dim]
    tol = 2e-6 if dtype == torch.complex64 else 1e-12
    for k in range(nt):
        r1 = t1(*X, c[k], nm[0] if dim == 1 else nm, eps=eps, isign=1)
        r2 = t2(*X, f[k], eps=eps, isign=-1)
        assert rel_l2(F[k].cpu().numpy(), r1.cpu().numpy()) <= tol
        assert rel_l2(C[k].cpu().numpy(), r2.cpu().numpy()) <= tol


def test_fft_same_plan_concurrent_streams():
    """One cached cuFFT plan launched on several streams at once (each stream with
    its own work area) gives every grid its own forward transform."""
    from nufftax_b200._plan import fft_inplace

    dev = cuda_device()
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    shape = (1, 16, 64, 1009)  # a prime axis (Bluestein)
    xs = [torch.complex(torch.randn(shape, device=dev, generator=g), torch.randn(shape, device=dev, generator=g))
          for _ in range(6)]
    refs = [torch.fft.fftn(x, dim=(-3, -2, -1)) for x in xs]
    ys = [x.clone() for x in xs]
    streams = [torch.cuda.Stream(dev) for _ in range(3)]
    torch.cuda.synchronize()
    for i, y in enumerate(ys):
        s = streams[i % 3]
        with torch.cuda.stream(s):
            fft_inplace(y, 3, -1)
    torch.cuda.synchronize()
    for y, r in zip(ys, refs):
        assert rel_l2(y.cpu().numpy(), r.cpu().numpy()) <= 1e-5


def test_fft_caller_work_area_and_capture():
    """nfx_fft_ws runs on a caller-owned work area (too small: NFX_ERR_WORKSPACE);
    a captured nfx_fft_ws replays correctly; nfx_fft refuses a capturing stream."""
    from ctypes import byref, c_size_t, c_void_p

    from nufftax_b200 import _lib
    from nufftax_b200._plan import fft_inplace, ptr

    dev = cuda_device()
    lib = _lib.load()
    nf = (150, 150, 90)
    nb_ = c_size_t(0)
    with torch.cuda.device(dev):
        assert lib.nfx_fft_work_bytes(_lib.NFX_F32, 3, _lib.int3(nf), 1, byref(nb_)) == 0
    assert nb_.value > 0
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    x = torch.complex(torch.randn((1,) + nf[::-1], device=dev, generator=g),
                      torch.randn((1,) + nf[::-1], device=dev, generator=g))
    ref = torch.fft.fftn(x, dim=(-3, -2, -1))
    work = torch.empty(nb_.value, dtype=torch.uint8, device=dev)
    y = x.clone()
    st = torch.cuda.current_stream(dev)
    assert lib.nfx_fft_ws(_lib.NFX_F32, 3, _lib.int3(nf), 1, ptr(y), -1, ptr(work), nb_.value - 1,
                          c_void_p(st.cuda_stream)) \
        == _lib.NFX_ERR_WORKSPACE
    assert lib.nfx_fft_ws(_lib.NFX_F32, 3, _lib.int3(nf), 1, ptr(y), -1, ptr(work), work.numel(),
                          c_void_p(st.cuda_stream)) == 0
    assert rel_l2(y.cpu().numpy(), ref.cpu().numpy()) <= 1e-5
    # captured: the graph keeps the caller's work area
    y.copy_(x)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    refused = None
    with torch.cuda.graph(graph):
        cs = torch.cuda.current_stream(dev)
        refused = lib.nfx_fft(_lib.NFX_F32, 3, _lib.int3(nf), 1, ptr(y), -1, c_void_p(cs.cuda_stream))
        assert lib.nfx_fft_ws(_lib.NFX_F32, 3, _lib.int3(nf), 1, ptr(y), -1, ptr(work), work.numel(),
                              c_void_p(cs.cuda_stream)) == 0
    assert refused == _lib.NFX_ERR_INVALID
    for _ in range(2):
        y.copy_(x)
        graph.replay()
        torch.cuda.synchronize()
        assert rel_l2(y.cpu().numpy(), ref.cpu().numpy()) <= 1e-5
    del graph
    # the per-stream path is unaffected
    y.copy_(x)
    fft_inplace(y, 3, -1)
    assert rel_l2(y.cpu().numpy(), ref.cpu().numpy()) <= 1e-5


def test_public_api_under_graph_capture():
    """nufft2d1 / nufft2d2 captured in a CUDA graph (the FFT takes its work area
    from the graph's pool; the sort made during capture stays out of the sort
    cache and is shared by the two transforms of the capture) replay to the
    eager results; an eager call after capture is unaffected."""
    dev = cuda_device()
    rng = np.random.default_rng(31)
    M, nm = 5000, (48, 40)
    x = torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev)
    y = torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev)
    c = torch.from_numpy((rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)).to(dev)
    f = torch.from_numpy((rng.standard_normal(nm[::-1]) + 1j * rng.standard_normal(nm[::-1])).astype(
        np.complex64)).to(dev)
    nb.sort_cache.clear()
    ref1 = nb.nufft2d1(x, y, c, nm).cpu().numpy()
    ref2 = nb.nufft2d2(x, y, f).cpu().numpy()
    nb.sort_cache.clear()
    xg, yg = x.clone(), y.clone()  # fresh tensors: no cached sort to reuse
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with profiling.record() as rec:
        with torch.cuda.graph(g):
            out1 = nb.nufft2d1(xg, yg, c, nm)
            out2 = nb.nufft2d2(xg, yg, f)
    # the type 2 reuses the sort captured for the type 1 (same capture, same stream)
    assert sum(1 for e in rec.events if e[0] == "nfx_sort_points") == 1
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        assert rel_l2(out1.cpu().numpy(), ref1) <= 1e-6
        assert rel_l2(out2.cpu().numpy(), ref2) <= 1e-6
    # eager on the same coordinates after capture sorts afresh
    assert rel_l2(nb.nufft2d1(xg, yg, c, nm).cpu().numpy(), ref1) <= 1e-6
    del g


def test_sort_shared_across_streams():
    """A type 1 on one stream and a type 2 on another on the same points share
    one sort: the second stream waits for the sort's completion event (eager),
    or joins it inside the graph (capture); both match the one-stream results."""
    dev = cuda_device()
    rng = np.random.default_rng(32)
    M, nm = 200_000, (96, 80)
    x = torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev)
    y = torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev)
    c = torch.from_numpy((rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)).to(dev)
    f = torch.from_numpy((rng.standard_normal(nm[::-1]) + 1j * rng.standard_normal(nm[::-1])).astype(
        np.complex64)).to(dev)
    nb.sort_cache.clear()
    ref1 = nb.nufft2d1(x, y, c, nm).cpu().numpy()
    ref2 = nb.nufft2d2(x, y, f).cpu().numpy()
    sa, sb = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def two_streams(xs, ys):
        cur = torch.cuda.current_stream(dev)
        sa.wait_stream(cur)
        sb.wait_stream(cur)
        with torch.cuda.stream(sa):
            o1 = nb.nufft2d1(xs, ys, c, nm)
        with torch.cuda.stream(sb):
            o2 = nb.nufft2d2(xs, ys, f)
        cur.wait_stream(sa)
        cur.wait_stream(sb)
        return o1, o2

    for rep in range(3):
        nb.sort_cache.clear()
        xs, ys = x.clone(), y.clone()
        with profiling.record() as rec:
            o1, o2 = two_streams(xs, ys)
        torch.cuda.synchronize()
        assert sum(1 for e in rec.events if e[0] == "nfx_sort_points") == 1
        assert rel_l2(o1.cpu().numpy(), ref1) <= 1e-6
        assert rel_l2(o2.cpu().numpy(), ref2) <= 1e-6
    nb.sort_cache.clear()
    xs, ys = x.clone(), y.clone()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with profiling.record() as rec:
        with torch.cuda.graph(g):
            o1, o2 = two_streams(xs, ys)
    assert sum(1 for e in rec.events if e[0] == "nfx_sort_points") == 1
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        assert rel_l2(o1.cpu().numpy(), ref1) <= 1e-6
        assert rel_l2(o2.cpu().numpy(), ref2) <= 1e-6
    del g


def test_malformed_request_fails_alone():
    """A request whose inputs do not match its description gets `error` set and no
    result; the requests around it complete correctly and the budget is released."""
    dev = cuda_device()
    rng = np.random.default_rng(12)
    reqs = _mix(rng, dev, n=8)
    bad = Request(kind=1, dim=2, n_modes=(16, 16), M=100,
                  coords=[torch.zeros(100, device=dev), torch.zeros(99, device=dev)],
                  strengths=torch.zeros(100, dtype=torch.complex64, device=dev))
    server = NufftServer(dev, slots=4, hbm_budget=2e9)
    done = server.serve(reqs[:4] + [bad] + reqs[4:])
    assert len(done) == 9 and server.in_use == 0
    assert bad.error is not None and bad.result is None
    for r in reqs:
        assert r.error is None
        assert rel_l2(r.result.cpu().numpy(), _alone(r).cpu().numpy()) <= 2e-6
    assert server.stats(done)["requests"] == 8


@pytest.mark.parametrize("dim,dtype", [(2, torch.complex64), (3, torch.complex64), (2, torch.complex128)])
def test_wave_entry_point_matches_api(dim, dtype):
    """nfx_wave: type-1 and type-2 problems of different grids and sizes in one
    call (one persistent spread and one interp launch) equal the public API
    transform by transform; the call is made twice with the same buffers."""
    from ctypes import byref, c_size_t, c_void_p

    from nufftax_b200 import _lib
    from nufftax_b200._plan import _facs, make_opts, ptr
    from nufftax_b200.grid import compute_grid_size
    from nufftax_b200.kernel import compute_kernel_params

    dev = cuda_device()
    rng = np.random.default_rng(40 + dim)
    eps = 1e-6 if dtype == torch.complex64 else 1e-9
    prec = _lib.NFX_F32 if dtype == torch.complex64 else _lib.NFX_F64
    rdt = torch.float32 if dtype == torch.complex64 else torch.float64
    kp = compute_kernel_params(eps)
    lib = _lib.load()
    n = 7
    items = (_lib.NfxWaveItem * n)()
    keep, probs = [], []
    common = None
    for i in range(n):
        kind = 1 + i % 2
        M = int(rng.integers(0 if i == 3 else 200, 20000))
        nm = tuple(int(rng.choice([12, 16, 24, 33])) for _ in range(dim))
        nf = tuple(compute_grid_size(v, 2.0, kp.nspread) for v in nm)
        o = make_opts(prec, nf, kp, prenorm=True)
        common = common or o
        X = [torch.from_numpy(rng.uniform(-np.pi, np.pi, M)).to(dev, rdt) for _ in range(dim)]
        if kind == 1:
            src = torch.from_numpy(rng.standard_normal(M) + 1j * rng.standard_normal(M)).to(dev, dtype)
            out = torch.empty(nm[::-1], dtype=dtype, device=dev)
        else:
            src = torch.from_numpy(rng.standard_normal(nm[::-1]) + 1j * rng.standard_normal(nm[::-1])).to(dev, dtype)
            out = torch.empty(M, dtype=dtype, device=dev)
        nb_ = c_size_t(0)
        assert lib.nfx_sort_workspace_bytes(byref(o), M, byref(nb_)) == 0
        ws = torch.empty(max(nb_.value, 1), dtype=torch.uint8, device=dev)
        fw = torch.empty(nf[::-1], dtype=dtype, device=dev)
        facs = _facs(nf, nm, kp, prec, dev)
        it = items[i]
        it.kind, it.M = kind, M
        cs = [x.data_ptr() for x in X] + [None] * (3 - dim)
        it.x, it.y, it.z = cs
        it.nf, it.n_modes = _lib.int3(nf), _lib.int3(nm)
        it.fft_sign = 1 if kind == 1 else -1
        it.fac = (c_void_p * 3)(*[f.data_ptr() if f is not None else None for f in facs])
        it.in_, it.out, it.fw = src.data_ptr(), out.data_ptr(), fw.data_ptr()
        it.workspace, it.workspace_bytes = ws.data_ptr(), ws.numel()
        keep += [X, src, out, ws, fw, facs]
        probs.append((kind, X, src, out, nm))
    tb = c_size_t(0)
    assert lib.nfx_wave_table_bytes(byref(common), items, n, byref(tb)) == 0, lib.nfx_last_error()
    table = torch.empty(tb.value, dtype=torch.uint8, device=dev)
    staging = torch.empty(tb.value, dtype=torch.uint8).pin_memory()
    st = c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    tol = 2e-6 if dtype == torch.complex64 else 1e-12
    for rep in range(2):
        assert lib.nfx_wave(byref(common), items, n, ptr(table), ptr(staging), table.numel(), st) == 0, \
            lib.nfx_last_error()
        torch.cuda.synchronize()
        for kind, X, src, out, nm in probs:
            if kind == 1:
                ref = {2: nb.nufft2d1, 3: nb.nufft3d1}[dim](*X, src, nm, eps=eps, isign=1)
            else:
                ref = {2: nb.nufft2d2, 3: nb.nufft3d2}[dim](*X, src, eps=eps, isign=-1)
            assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) <= tol or (X[0].numel() == 0)
