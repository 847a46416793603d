"""GPU: the no-allocation spreading entry point (nfx_spread_noalloc).

Some callers cannot allocate device memory or hand over a workspace, for
example code running inside another framework's operator that only receives
its operand and result buffers.  nfx_spread_noalloc serves them from a fixed
scratch array inside the library.  These tests call it through the C ABI and
compare it with nfx_spread (same kernels, caller workspace) within the
complex64 spread tolerance used elsewhere (relative l2 <= 2e-6), on two calls
in a row, and check that an oversized request is refused.  The file name makes
pytest collect it last.
"""

import ctypes
from ctypes import byref, c_size_t, c_void_p

import numpy as np
import pytest
import torch

import nufftax_b200 as nb
from nufftax_b200 import _lib
from nufftax_b200._plan import make_opts
from tests.conftest import cuda_device, rel_l2

pytestmark = pytest.mark.gpu


def _spread_pair(lib, dev, rng, M, nf):
    kp = nb.compute_kernel_params(1e-6)
    opts = make_opts(_lib.NFX_F32, nf, kp, prenorm=True)
    x = torch.from_numpy(rng.uniform(-np.pi, np.pi, M).astype(np.float32)).to(dev)
    y = torch.from_numpy((0.3 * rng.standard_normal(M)).astype(np.float32)).to(dev)
    c = torch.from_numpy((rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))).astype(np.complex64)).to(dev)
    shape = (2, nf[1], nf[0])
    stream = c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    want = torch.empty(shape, dtype=torch.complex64, device=dev)
    nbytes = c_size_t(0)
    assert lib.nfx_sort_workspace_bytes(byref(opts), M, byref(nbytes)) == 0
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    assert lib.nfx_spread(byref(opts), c_void_p(x.data_ptr()), c_void_p(y.data_ptr()), None, M,
                          c_void_p(c.data_ptr()), 2, c_void_p(want.data_ptr()), c_void_p(ws.data_ptr()),
                          nbytes.value, stream) == 0
    got = torch.full(shape, complex(7.0, -7.0), dtype=torch.complex64, device=dev)
    st = lib.nfx_spread_noalloc(byref(opts), c_void_p(x.data_ptr()), c_void_p(y.data_ptr()), None, M,
                                c_void_p(c.data_ptr()), 2, c_void_p(got.data_ptr()), stream)
    assert st == 0, lib.nfx_last_error()
    torch.cuda.synchronize(dev)
    return got.cpu().numpy(), want.cpu().numpy()


def test_noalloc_matches_workspace_entry_point_twice():
    dev = cuda_device()
    lib = _lib.load()
    rng = np.random.default_rng(2026)
    # two calls in a row on different sizes: the second must not see the first's leftovers
    for M, nf in ((300_000, (256, 192)), (70_000, (96, 128))):
        got, want = _spread_pair(lib, dev, rng, M, nf)
        assert rel_l2(got, want) <= 2e-6


def test_noalloc_rejects_oversized_request():
    dev = cuda_device()
    lib = _lib.load()
    kp = nb.compute_kernel_params(1e-6)
    opts = make_opts(_lib.NFX_F32, (1024, 1024), kp, prenorm=True)
    cap = lib.nfx_noalloc_scratch_bytes()
    assert cap == 64 << 20
    M = 20_000_000
    nbytes = c_size_t(0)
    assert lib.nfx_sort_workspace_bytes(byref(opts), M, byref(nbytes)) == 0
    assert nbytes.value > cap
    fw = torch.empty(1, dtype=torch.complex64, device=dev)
    st = lib.nfx_spread_noalloc(byref(opts), c_void_p(8), c_void_p(8), None, M, c_void_p(8), 1,
                                c_void_p(fw.data_ptr()), None)
    assert st == _lib.NFX_ERR_UNSUPPORTED
    assert b"scratch" in lib.nfx_last_error()
