"""GPU: the interpolation's TMA tile staging.

Interior tiles are copied by one cp.async.bulk.tensor box load, wrapping tiles
by plain loads; NFX_INTERP_STAGING=plain forces plain loads everywhere.  Both
stagings put the same values in the same shared-memory layout, so the outputs
must be bit-identical, over tilings that do and do not qualify for TMA (odd
tile edges, odd fine-grid rows, tiles as large as the grid, several
transforms, complex128), and the device status word must stay 0 (no bounded
wait gave up).  The TMA result is also checked against the oracle.
"""

import os

import numpy as np
import pytest
import torch

from nufftax_b200 import _lib
from nufftax_b200._plan import PointSort
from nufftax_b200.kernel import compute_kernel_params
from oracle import nufft_oracle as O
from tests.conftest import cuda_device, rel_l2

pytestmark = pytest.mark.gpu


def _interp_both(ps, fw):
    old = os.environ.get("NFX_INTERP_STAGING")
    try:
        os.environ["NFX_INTERP_STAGING"] = "plain"
        plain = ps.interp(fw).clone()
        os.environ.pop("NFX_INTERP_STAGING")
        tma = ps.interp(fw).clone()
    finally:
        if old is None:
            os.environ.pop("NFX_INTERP_STAGING", None)
        else:
            os.environ["NFX_INTERP_STAGING"] = old
    return plain, tma


CASES = [
    # dim, nf, tile, M, n_trans, dtype, clustered
    (2, (256, 192), None, 60_000, 1, np.float32, True),
    (2, (256, 192), (15, 17), 60_000, 1, np.float32, False),   # odd x edge: plain loads only
    (2, (250, 130), (32, 16), 40_000, 2, np.float32, False),   # grid edge not a tile multiple
    (2, (64, 64), (64, 64), 5_000, 1, np.float32, False),      # one tile covers the grid: always wraps
    (2, (200, 96), None, 30_000, 3, np.float64, True),
    (3, (48, 40, 36), None, 80_000, 1, np.float32, False),
    (3, (48, 40, 36), (8, 8, 8), 80_000, 2, np.float32, True),
    (3, (32, 32, 32), None, 20_000, 1, np.float64, False),
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("mode", [_lib.NFX_PER_POINT_THREAD, _lib.NFX_PER_POINT_GROUP])
def test_tma_staging_bit_identical(case, mode):
    dim, nf, tile, M, ntr, dt, clustered = CASES[case]
    dev = cuda_device()
    rng = np.random.default_rng(100 + case)
    if clustered:
        X = [np.mod(0.4 * rng.standard_normal(M) + np.pi, 2 * np.pi) - np.pi for _ in range(dim)]
    else:
        X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
    X = [x.astype(dt) for x in X]
    eps = 1e-6 if dt == np.float32 else 1e-10
    kp = compute_kernel_params(eps, 2.0)
    cdt = np.complex64 if dt == np.float32 else np.complex128
    shape = (ntr,) + tuple(reversed(nf))
    fw_np = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(cdt)
    Xt = [torch.from_numpy(x).to(dev) for x in X]
    fw = torch.from_numpy(fw_np).to(dev)
    ps = PointSort(Xt, nf, kp, prenorm=True, tile=tile, modes=(0, mode))
    assert _lib.device_status() == 0
    plain, tma = _interp_both(ps, fw)
    assert _lib.device_status() == 0
    assert torch.equal(plain, tma)
    # the TMA-staged result against the oracle's interpolation
    sel = slice(0, min(M, 4000))
    ref = O.interp([x[sel] for x in X], fw_np, kp)
    got = tma.cpu().numpy()[..., sel]
    tol = 1e-5 if dt == np.float32 else 1e-11
    assert rel_l2(got.reshape(ref.shape), ref) <= tol


def test_bounded_wait_gives_up_and_reports():
    """The tile-copy wait is bounded: a barrier armed for a copy that is never
    issued (nfx_selftest_bounded_wait) makes the kernel give up, record
    NFX_STATUS_TMA_TIMEOUT and return; the context stays usable and the status
    reads clean again afterwards."""
    import ctypes

    lib = _lib.load()
    assert _lib.device_status() == 0
    st = ctypes.c_int(0)
    _lib.check(lib.nfx_selftest_bounded_wait(ctypes.byref(st)), "nfx_selftest_bounded_wait")
    assert st.value == _lib.NFX_STATUS_TMA_TIMEOUT
    assert _lib.device_status() == 0
    # the device still runs the path afterwards
    dev = cuda_device()
    rng = np.random.default_rng(7)
    X = [rng.uniform(-np.pi, np.pi, 3000).astype(np.float32) for _ in range(2)]
    kp = compute_kernel_params(1e-6, 2.0)
    fw_np = (rng.standard_normal((1, 96, 128)) + 1j * rng.standard_normal((1, 96, 128))).astype(np.complex64)
    ps = PointSort([torch.from_numpy(x).to(dev) for x in X], (128, 96), kp, prenorm=True)
    got = ps.interp(torch.from_numpy(fw_np).to(dev)).cpu().numpy()
    ref = O.interp(X, fw_np, kp)
    assert rel_l2(got.reshape(ref.shape), ref) <= 1e-5
    assert _lib.device_status() == 0


@pytest.mark.parametrize("case", [0, 2, 4, 5, 6, 7])
def test_tma_staging_gradient_pass_bit_identical(case):
    """The fused gradient pass (value + coordinate gradients, both adjoints)
    stages its tile the same way: TMA and plain staging give identical outputs."""
    dim, nf, tile, M, ntr, dt, clustered = CASES[case]
    dev = cuda_device()
    rng = np.random.default_rng(200 + case)
    X = [rng.uniform(-np.pi, np.pi, M).astype(dt) for _ in range(dim)]
    kp = compute_kernel_params(1e-6 if dt == np.float32 else 1e-10, 2.0)
    cdt = np.complex64 if dt == np.float32 else np.complex128
    shape = (ntr,) + tuple(reversed(nf))
    G = torch.from_numpy((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(cdt)).to(dev)
    c = torch.from_numpy((rng.standard_normal((ntr, M)) + 1j * rng.standard_normal((ntr, M))).astype(cdt)).to(dev)
    ps = PointSort([torch.from_numpy(x).to(dev) for x in X], nf, kp, prenorm=True, tile=tile)
    need = [True] * dim

    def both():
        dc, dxs = ps.spread_grad(c, G, True, need)
        ixs = ps.interp_grad(G, c, need)
        return [dc.clone()] + [d.clone() for d in dxs] + [d.clone() for d in ixs]

    old = os.environ.get("NFX_INTERP_STAGING")
    try:
        os.environ["NFX_INTERP_STAGING"] = "plain"
        plain = both()
        os.environ.pop("NFX_INTERP_STAGING")
        tma = both()
    finally:
        if old is not None:
            os.environ["NFX_INTERP_STAGING"] = old
    assert _lib.device_status() == 0
    for p_, t_ in zip(plain, tma):
        assert torch.equal(p_, t_)
