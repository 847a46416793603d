"""GPU: the continuous-batching server returns, for every request of a mixed
stream served concurrently, the same result as the request alone through the
public API (relative l2 <= 2 eps, eps = 1e-6), and honours its memory budget."""

import numpy as np
import pytest
import torch

import nufftax_b200 as nb
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
