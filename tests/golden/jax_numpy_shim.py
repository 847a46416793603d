"""A NumPy stand-in for the part of the jax API that nufftax's pure-JAX path uses.

TEST INFRASTRUCTURE ONLY, used by make_reference_golden.py in a container that
holds the reference source but no jax.  Installing it (`install()`) puts modules
named `jax`, `jax.numpy`, `jax.ops` and `jax.lax` in sys.modules, so that the
reference's own modules (nufftax/core/*.py, nufftax/utils/grid.py,
nufftax/transforms/nufft{1,2,3}.py) import and run unmodified on NumPy:

  * arrays are NumPy arrays with JAX's functional update syntax
    (`a.at[idx].set(v)` / `.add(v)` return updated copies);
  * `jax.numpy` forwards to NumPy (NumPy 2 treats Python scalars as weakly
    typed, as JAX does, so float32 inputs keep float32 arithmetic; its FFTs of
    complex64 arrays compute in single precision);
  * `jax.jit` returns the function unchanged, `jax.custom_vjp` calls the primal
    function (its fwd/bwd rules stay reachable as plain functions),
    `jax.vmap` maps over an axis with a Python loop;
  * `jax.ops.segment_sum` accumulates with `numpy.add.at` in the data's dtype;
  * `jax.config.jax_enable_x64` is True, the configuration nufftax's own tests
    run in (tests/conftest.py:30), so default dtypes are 64-bit as in NumPy;
  * `jax.devices()` reports one CPU device (the Pallas path stays off).

What it does not reproduce: XLA's operation fusion and the accumulation order of
its scatter-add, so results agree with a real JAX run to float rounding, not
bit for bit, except where the reference's float arithmetic is elementwise
(coordinate folding), where NumPy performs the same IEEE operations.
"""

from __future__ import annotations

import sys
import types

import numpy as np


class Array(np.ndarray):
    """NumPy array with JAX's `.at[...]` functional updates."""

    @property
    def at(self):
        return _At(self)


class _At:
    def __init__(self, a):
        self._a = a

    def __getitem__(self, idx):
        return _AtIndex(self._a, idx)


class _AtIndex:
    def __init__(self, a, idx):
        self._a = a
        self._idx = idx

    def _copy(self):
        return np.array(self._a, copy=True).view(Array)

    def set(self, v):
        out = self._copy()
        out[self._idx] = v
        return out

    def add(self, v):
        out = self._copy()
        np.add.at(out, self._idx, v)
        return out

    def multiply(self, v):
        out = self._copy()
        np.multiply.at(out, self._idx, v)
        return out

    def get(self):
        return _wrap(self._a[self._idx])


def _wrap(r):
    if isinstance(r, np.ndarray) and not isinstance(r, Array):
        return r.view(Array)
    if isinstance(r, tuple):
        return tuple(_wrap(v) for v in r)
    if isinstance(r, list):
        return [_wrap(v) for v in r]
    return r


def _wrapped(fn):
    def call(*args, **kwargs):
        return _wrap(fn(*args, **kwargs))

    call.__name__ = getattr(fn, "__name__", "fn")
    return call


class _NumpyModule(types.ModuleType):
    """Module whose attributes come from a NumPy namespace, results as Array."""

    def __init__(self, name, base):
        super().__init__(name)
        self._base = base

    def __getattr__(self, name):
        v = getattr(self._base, name)
        if callable(v) and not isinstance(v, type):
            v = _wrapped(v)
        setattr(self, name, v)
        return v


def _array(obj, dtype=None, copy=True, **kw):
    return np.array(obj, dtype=dtype, copy=copy).view(Array)


def _asarray(obj, dtype=None, **kw):
    return np.asarray(obj, dtype=dtype).view(Array)


def jit(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


class custom_vjp:
    """Calls the primal function; defvjp records the rules (not applied)."""

    def __init__(self, fun, nondiff_argnums=()):
        self.fun = fun
        self.nondiff_argnums = nondiff_argnums
        self.fwd = self.bwd = None

    def defvjp(self, fwd, bwd):
        self.fwd, self.bwd = fwd, bwd

    def __call__(self, *args, **kwargs):
        return self.fun(*args, **kwargs)


class custom_jvp(custom_vjp):
    def defjvp(self, jvp):
        self.jvp = jvp


def vmap(fun, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = next(np.shape(a)[ax] for a, ax in zip(args, axes) if ax is not None)
        outs = []
        for i in range(n):
            outs.append(fun(*[a if ax is None else np.take(a, i, axis=ax) for a, ax in zip(args, axes)]))
        if isinstance(outs[0], tuple):
            return tuple(_wrap(np.stack([o[k] for o in outs], axis=out_axes)) for k in range(len(outs[0])))
        return _wrap(np.stack(outs, axis=out_axes))

    return mapped


def segment_sum(data, segment_ids, num_segments=None, indices_are_sorted=False, unique_indices=False, **kw):
    data = np.asarray(data)
    ids = np.asarray(segment_ids)
    n = int(num_segments) if num_segments is not None else int(ids.max()) + 1
    out = np.zeros((n,) + data.shape[1:], dtype=data.dtype)
    np.add.at(out, ids, data)
    return out.view(Array)


class _Device:
    platform = "cpu"


def devices(*args):
    return [_Device()]


class _Config:
    jax_enable_x64 = True

    def update(self, name, value):
        setattr(self, name, value)


def install():
    """Register the stand-in as `jax` (only when no real jax is importable)."""
    try:
        import jax  # noqa: F401

        raise RuntimeError("a real jax is importable: use it instead of the stand-in")
    except ImportError:
        pass
    jax = types.ModuleType("jax")
    jnp = _NumpyModule("jax.numpy", np)
    jnp.array = _array
    jnp.asarray = _asarray
    jnp.ndarray = Array
    jnp.fft = _NumpyModule("jax.numpy.fft", np.fft)
    ops = types.ModuleType("jax.ops")
    ops.segment_sum = segment_sum
    lax = types.ModuleType("jax.lax")
    jax.numpy = jnp
    jax.ops = ops
    jax.lax = lax
    jax.Array = Array
    jax.jit = jit
    jax.custom_vjp = custom_vjp
    jax.custom_jvp = custom_jvp
    jax.vmap = vmap
    jax.devices = devices
    jax.config = _Config()
    sys.modules.update({"jax": jax, "jax.numpy": jnp, "jax.numpy.fft": jnp.fft, "jax.ops": ops, "jax.lax": lax})
    return jax


def import_reference(root):
    """Import the reference's pure-JAX modules from `root` (the nufftax project
    root) without its package __init__ files that pull in the JAX primitive
    machinery: returns a namespace with core.kernel, core.spread,
    core.deconvolve, utils.grid and transforms.nufft1/2/3."""
    import importlib

    install()
    pkg_dir = f"{root}/nufftax"
    for name, sub in (("nufftax", ""), ("nufftax.transforms", "/transforms")):
        m = types.ModuleType(name)
        m.__path__ = [pkg_dir + sub]
        sys.modules[name] = m
    ns = types.SimpleNamespace()
    for mod in ("core.kernel", "core.spread", "core.deconvolve", "utils.grid", "transforms.nufft1",
                "transforms.nufft2", "transforms.nufft3"):
        setattr(ns, mod.replace(".", "_"), importlib.import_module("nufftax." + mod))
    return ns
