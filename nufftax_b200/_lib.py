"""ctypes binding of libnfx_b200.so (the C ABI declared in include/nfx.h).

The library is required: importing the compute entry points without it raises,
there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import re
import threading
from ctypes import POINTER, c_double, c_int, c_int64, c_size_t, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).with_name("libnfx_b200.so")
HEADER_PATH = Path(__file__).resolve().parent.parent / "include" / "nfx.h"

NFX_OK = 0
NFX_ERR_INVALID = 1
NFX_ERR_WORKSPACE = 2
NFX_ERR_CUDA = 3
NFX_ERR_CUFFT = 4
NFX_ERR_UNSUPPORTED = 5
NFX_F32 = 0
NFX_F64 = 1
# threads per point of the spread / interpolation (nfx_opts::spread_mode, interp_mode)
NFX_PER_POINT_AUTO = 0
NFX_PER_POINT_THREAD = 1
NFX_PER_POINT_GROUP = 2
NFX_PER_POINT_WARP = 3
NFX_PER_POINT_CTA = 4
NFX_STATUS_TMA_TIMEOUT = 1

_STATUS = {
    NFX_ERR_INVALID: ValueError,
    NFX_ERR_WORKSPACE: ValueError,
    NFX_ERR_UNSUPPORTED: NotImplementedError,
}


class NfxError(RuntimeError):
    """A CUDA or cuFFT failure reported by libnfx_b200."""


class NfxOpts(ctypes.Structure):
    """Mirror of `nfx_opts` in include/nfx.h."""

    _fields_ = [
        ("precision", c_int),
        ("dim", c_int),
        ("nf", c_int * 3),
        ("nspread", c_int),
        ("beta", c_double),
        ("kc", c_double),
        ("prenorm", c_int),
        ("tile", c_int * 3),
        ("max_subproblem", c_int),
        ("spread_mode", c_int),
        ("interp_mode", c_int),
    ]


class NfxBatchProblem(ctypes.Structure):
    """Mirror of `nfx_batch_problem` in include/nfx.h."""

    _fields_ = [
        ("M", c_int64),
        ("x", c_void_p),
        ("y", c_void_p),
        ("z", c_void_p),
        ("nf", c_int * 3),
        ("tile", c_int * 3),
        ("max_subproblem", c_int),
        ("interp_mode", c_int),
        ("workspace", c_void_p),
        ("workspace_bytes", c_size_t),
        ("src", c_void_p),
        ("dst", c_void_p),
    ]


class NfxWaveItem(ctypes.Structure):
    """Mirror of `nfx_wave_item` in include/nfx.h."""

    _fields_ = [
        ("kind", c_int),
        ("M", c_int64),
        ("x", c_void_p),
        ("y", c_void_p),
        ("z", c_void_p),
        ("nf", c_int * 3),
        ("n_modes", c_int * 3),
        ("fft_sign", c_int),
        ("fac", c_void_p * 3),
        ("in_", c_void_p),
        ("out", c_void_p),
        ("fw", c_void_p),
        ("workspace", c_void_p),
        ("workspace_bytes", c_size_t),
    ]


class NfxBatchInfo(ctypes.Structure):
    """Mirror of `nfx_batch_info` in include/nfx.h."""

    _fields_ = [("table_bytes", c_size_t), ("smem_bytes", c_size_t), ("max_subs", c_int64)]


_vp = c_void_p
_SIGNATURES = {
    "nfx_version": ([], c_int),
    "nfx_last_error": ([], ctypes.c_char_p),
    "nfx_num_sms": ([], c_int),
    "nfx_device_status": ([POINTER(c_int)], c_int),
    "nfx_selftest_bounded_wait": ([POINTER(c_int)], c_int),
    "nfx_capture_id": ([c_void_p, POINTER(ctypes.c_ulonglong)], c_int),
    "nfx_sort_kernel_count": ([POINTER(NfxOpts), c_int64, c_int, POINTER(c_int)], c_int),
    "nfx_es_poly": ([c_int, c_double, c_double, POINTER(ctypes.c_float), POINTER(c_int), POINTER(c_double)], c_int),
    "nfx_default_tiles": ([POINTER(NfxOpts)], c_int),
    "nfx_sort_workspace_bytes": ([POINTER(NfxOpts), c_int64, POINTER(c_size_t)], c_int),
    "nfx_sort_points": ([POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, c_size_t, _vp], c_int),
    "nfx_sort_results": ([POINTER(NfxOpts), c_int64, _vp, c_size_t, _vp, _vp, _vp, POINTER(c_int), _vp], c_int),
    "nfx_spread": ([POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, c_int, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_interp": ([POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, c_int, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_noalloc_scratch_bytes": ([], c_size_t),
    "nfx_spread_noalloc": ([POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, c_int, _vp, _vp], c_int),
    "nfx_spread_sorted": ([POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, c_int, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_interp_sorted": ([POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, c_int, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_spread_grad_sorted": (
        [POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, _vp, c_int, _vp, _vp, _vp, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_interp_grad_sorted": (
        [POINTER(NfxOpts), _vp, _vp, _vp, c_int64, _vp, _vp, c_int, _vp, _vp, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_deconv_shuffle": ([c_int, c_int, POINTER(c_int), POINTER(c_int), _vp, _vp, _vp, _vp, _vp, c_int, _vp],
                           c_int),
    "nfx_deconv_pad": ([c_int, c_int, POINTER(c_int), POINTER(c_int), _vp, _vp, _vp, _vp, _vp, c_int, _vp], c_int),
    "nfx_fft": ([c_int, c_int, POINTER(c_int), c_int, _vp, c_int, _vp], c_int),
    "nfx_fft_work_bytes": ([c_int, c_int, POINTER(c_int), c_int, POINTER(c_size_t)], c_int),
    "nfx_fft_ws": ([c_int, c_int, POINTER(c_int), c_int, _vp, c_int, _vp, c_size_t, _vp], c_int),
    "nfx_nufft1": ([POINTER(NfxOpts), POINTER(c_int), _vp, _vp, _vp, c_int64, _vp, c_int, c_int, _vp, _vp, _vp, _vp,
                    _vp, _vp, c_size_t, _vp], c_int),
    "nfx_nufft2": ([POINTER(NfxOpts), POINTER(c_int), _vp, _vp, _vp, c_int64, _vp, c_int, c_int, _vp, _vp, _vp, _vp,
                    _vp, _vp, c_size_t, _vp], c_int),
    "nfx_fft_cache_clear": ([], c_int),
    "nfx_fft_cache_limit": ([c_int], c_int),
    "nfx_batch_info_get": ([POINTER(NfxOpts), c_int, POINTER(NfxBatchProblem), c_int, POINTER(NfxBatchInfo)], c_int),
    "nfx_batch_upload": ([POINTER(NfxOpts), c_int, POINTER(NfxBatchProblem), c_int, _vp, c_size_t, _vp], c_int),
    "nfx_batch_sort": ([POINTER(NfxOpts), POINTER(NfxBatchProblem), c_int, _vp], c_int),
    "nfx_batch_launch": ([POINTER(NfxOpts), c_int, _vp, c_int, POINTER(NfxBatchInfo), _vp], c_int),
    "nfx_batch_deconv_table_bytes": ([c_int, c_int], c_size_t),
    "nfx_batch_deconv_upload": ([c_int, c_int, c_int, POINTER(c_int), POINTER(c_int), POINTER(c_void_p),
                                 POINTER(c_void_p), POINTER(c_void_p), c_int, _vp, c_size_t, POINTER(c_int64), _vp],
                                c_int),
    "nfx_batch_deconv": ([c_int, c_int, _vp, c_int, c_int64, _vp], c_int),
    "nfx_wave_table_bytes": ([POINTER(NfxOpts), POINTER(NfxWaveItem), c_int, POINTER(c_size_t)], c_int),
    "nfx_wave": ([POINTER(NfxOpts), POINTER(NfxWaveItem), c_int, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_nufft3_workspace_bytes": ([POINTER(NfxOpts), POINTER(c_int), c_int64, c_int64, c_int, POINTER(c_size_t)],
                                   c_int),
    "nfx_nufft3": ([POINTER(NfxOpts), POINTER(c_int), c_double, c_int, POINTER(c_void_p), c_int64, _vp, c_int,
                    POINTER(c_void_p), c_int64, _vp, _vp, _vp, _vp, _vp, c_size_t, _vp], c_int),
    "nfx_t3_params_bytes": ([], c_size_t),
    "nfx_t3_scratch_bytes": ([c_int, c_int64, c_int64], c_size_t),
    "nfx_t3_prepare": ([c_int, c_int, POINTER(c_int), c_int, c_double, c_double, c_double, c_int, POINTER(c_void_p),
                        c_int64, _vp, c_int, POINTER(c_void_p), c_int64, _vp, POINTER(c_void_p), _vp,
                        POINTER(c_void_p), _vp, _vp, c_size_t, _vp], c_int),
    "nfx_t3_finish": ([c_int, _vp, c_int64, c_int, _vp, _vp], c_int),
}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def header_symbols() -> list[str]:
    """Function names declared in include/nfx.h."""
    text = HEADER_PATH.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\**\s+\**(nfx_[a-z0-9_]+)\s*\(", text, re.M)))


def load() -> ctypes.CDLL:
    """Load libnfx_b200.so once and attach argument types; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python -m nufftax_b200._build` (nvcc, sm_100a). "
                "nufftax_b200 has no CPU fallback.")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


def check(status: int, what: str) -> None:
    """Raise the Python exception matching an nfx status code."""
    if status == NFX_OK:
        return
    msg = load().nfx_last_error().decode(errors="replace")
    exc = _STATUS.get(status, NfxError)
    raise exc(f"{what} failed (nfx status {status}): {msg}")


def int3(vals) -> ctypes.Array:
    arr = (c_int * 3)(1, 1, 1)
    for i, v in enumerate(vals):
        arr[i] = int(v)
    return arr


_int3_cache: dict = {}


def int3c(vals) -> ctypes.Array:
    """int3 for read-only arguments (`const int[3]`), shared per value: the hot
    paths pass the same grid sizes on every call."""
    key = tuple(int(v) for v in vals)
    arr = _int3_cache.get(key)
    if arr is None:
        if len(_int3_cache) >= 4096:
            _int3_cache.clear()
        arr = _int3_cache[key] = int3(key)
    return arr


def device_status() -> int:
    """Status bits of the current GPU (NFX_STATUS_*; 0 when no bounded wait in
    a kernel gave up), cleared by the read.  Synchronizes the device."""
    st = c_int(0)
    check(load().nfx_device_status(ctypes.byref(st)), "nfx_device_status")
    return int(st.value)
