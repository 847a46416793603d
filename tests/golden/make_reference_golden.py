"""Golden vectors computed by the reference's own source (nufftax v0.6.0).

Run in a container that holds the reference checkout (its path is the only
argument; default /root/reference) and no jax:

    python tests/golden/make_reference_golden.py /root/reference

The reference's pure-JAX modules (nufftax/core/{kernel,spread,deconvolve}.py,
nufftax/utils/grid.py, nufftax/transforms/nufft{1,2,3}.py) are imported
unmodified and run on NumPy through jax_numpy_shim.py, in the configuration of
nufftax's own tests (jax_enable_x64 on, tests/conftest.py:30).  Seeded inputs
and the reference's outputs go to tests/golden/ref_*.npz:

  ref_fold.npz       fold_rescale (spread.py:78-97) and the transforms'
                     pre-normalisation jnp.mod(x + pi, 2 pi) - pi on float32
                     and float64 inputs with folding edge cases (bit-exact:
                     elementwise IEEE operations);
  ref_t{1,2,3}.npz   nufft{1,2,3}d{1,2,3} over dims, precisions, eps, isign,
                     n_trans and upsampfac;
  ref_core.npz       spread_{2,3}d / interp_{2,3}d and their custom_vjp
                     backward rules (spread.py:952-1305) for real-valued
                     strengths, where JAX's and torch's complex cotangent
                     conventions coincide.

A real jax would accumulate the float32 scatter-adds in another order, so the
complex64 vectors pin the reference to float rounding (~1e-7 relative); the
complex128 ones to ~1e-15.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import jax_numpy_shim  # noqa: E402

T1_CASES = [  # (dim, n_modes, M, precision, eps, isign, upsampfac, n_trans)
    (1, (64,), 1000, "c64", 1e-6, 1, 2.0, 0),
    (1, (257,), 3000, "c128", 1e-12, -1, 2.0, 2),
    (2, (32, 24), 2000, "c64", 1e-6, 1, 2.0, 0),
    (2, (33, 20), 2500, "c128", 1e-9, -1, 2.0, 0),
    (2, (40, 30), 1500, "c64", 1e-6, 1, 1.25, 0),
    (3, (16, 12, 10), 2000, "c64", 1e-6, 1, 2.0, 0),
    (3, (12, 9, 8), 1500, "c128", 1e-12, -1, 2.0, 2),
]
T3_CASES = [  # (dim, M, K, s_extent, precision, eps, isign, n_trans)
    (1, 400, 300, 30.0, "c64", 1e-6, 1, 0),
    (2, 500, 400, 20.0, "c64", 1e-6, 1, 0),
    (2, 500, 300, 25.0, "c128", 1e-9, -1, 2),
    (3, 300, 250, 8.0, "c128", 1e-12, 1, 0),
]


def _dt(prec):
    return (np.float32, np.complex64) if prec == "c64" else (np.float64, np.complex128)


def _cplx(rng, shape, dt):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dt)


def _key(case):
    return "_".join(str(v).replace(" ", "").replace(",", "x").replace("(", "").replace(")", "") for v in case)


def make(root: str) -> None:
    R = jax_numpy_shim.import_reference(root)
    n1, n2, n3 = R.transforms_nufft1, R.transforms_nufft2, R.transforms_nufft3
    rng = np.random.default_rng(20240601)

    # -- folding ----------------------------------------------------------------
    edge = np.array([np.pi, -np.pi, 0.0, 3.5, -3.5, 7.0, -1e-8, 1e-8, 2 * np.pi, -2 * np.pi, 1e4, -1e4, 3.14159,
                     -3.14159, 1e-30])
    fold = {}
    for name, dt in (("f32", np.float32), ("f64", np.float64)):
        x = np.concatenate([edge, rng.uniform(-np.pi, np.pi, 2000), rng.uniform(-20, 20, 500)]).astype(dt)
        x = np.concatenate([x, np.nextafter(x[:15], np.array(np.inf, dt)), np.nextafter(x[:15], np.array(-np.inf, dt))])
        pre = np.asarray(np.mod(x + np.pi, 2.0 * np.pi) - np.pi)  # nufft1.py:71, the same jnp ops
        fold[f"x_{name}"] = x
        fold[f"premod_{name}"] = np.asarray(R.core_spread.jnp.mod(x + R.core_spread.jnp.pi, 2.0 * R.core_spread.jnp.pi)
                                            - R.core_spread.jnp.pi)
        assert np.array_equal(fold[f"premod_{name}"], pre)
        for nf in (16384, 1024, 250, 7):
            fold[f"fold_{name}_{nf}"] = np.asarray(R.core_spread.fold_rescale(fold[f"premod_{name}"], nf))
    np.savez_compressed(HERE / "ref_fold.npz", **fold)

    # -- types 1 and 2 ------------------------------------------------------------
    fn1 = {1: n1.nufft1d1, 2: n1.nufft2d1, 3: n1.nufft3d1}
    fn2 = {1: n2.nufft1d2, 2: n2.nufft2d2, 3: n2.nufft3d2}
    t1, t2 = {}, {}
    for case in T1_CASES:
        dim, nm, M, prec, eps, isign, uf, nt = case
        rdt, cdt = _dt(prec)
        X = [rng.uniform(-np.pi, np.pi, M).astype(rdt) for _ in range(dim)]
        c = _cplx(rng, (nt, M) if nt else M, cdt)
        f = _cplx(rng, ((nt,) if nt else ()) + tuple(reversed(nm)), cdt)
        modes = nm[0] if dim == 1 else nm
        k = _key(case)
        for d in range(dim):
            t1[f"{k}/x{d}"] = X[d]
        t1[f"{k}/c"] = c
        t1[f"{k}/out"] = np.asarray(fn1[dim](*X, c, modes, eps=eps, isign=isign, upsampfac=uf))
        for d in range(dim):
            t2[f"{k}/x{d}"] = X[d]
        t2[f"{k}/f"] = f
        t2[f"{k}/out"] = np.asarray(fn2[dim](*X, f, eps=eps, isign=-isign, upsampfac=uf))
    np.savez_compressed(HERE / "ref_t1.npz", **t1)
    np.savez_compressed(HERE / "ref_t2.npz", **t2)

    # -- type 3 ---------------------------------------------------------------------
    fn3 = {1: n3.nufft1d3, 2: n3.nufft2d3, 3: n3.nufft3d3}
    t3 = {}
    for case in T3_CASES:
        dim, M, K, S, prec, eps, isign, nt = case
        rdt, cdt = _dt(prec)
        X = [rng.uniform(-np.pi, np.pi, M).astype(rdt) for _ in range(dim)]
        T = [rng.uniform(-S, S, K).astype(rdt) for _ in range(dim)]
        c = _cplx(rng, (nt, M) if nt else M, cdt)
        if dim == 1:
            nf = (n3.compute_type3_grid_size(X[0], T[0], eps=eps),)
            out = fn3[1](X[0], c, T[0], nf[0], eps=eps, isign=isign)
        elif dim == 2:
            nf = n3.compute_type3_grid_sizes_2d(np.pi, np.pi, S, S, eps=eps)
            out = fn3[2](X[0], X[1], c, T[0], T[1], nf, eps=eps, isign=isign)
        else:
            nf = n3.compute_type3_grid_sizes_3d(np.pi, np.pi, np.pi, S, S, S, eps=eps)
            out = fn3[3](X[0], X[1], X[2], c, T[0], T[1], T[2], nf, eps=eps, isign=isign)
        k = _key(case)
        for d in range(dim):
            t3[f"{k}/x{d}"] = X[d]
            t3[f"{k}/s{d}"] = T[d]
        t3[f"{k}/c"] = c
        t3[f"{k}/nf"] = np.asarray(nf)
        t3[f"{k}/out"] = np.asarray(out)
    np.savez_compressed(HERE / "ref_t3.npz", **t3)

    # -- core spread / interp and their backward rules ------------------------------
    core = {}
    sp = R.core_spread
    kp = R.core_kernel.compute_kernel_params(1e-9)
    for dim, nf, M in ((2, (40, 36), 1200), (3, (20, 18, 16), 900)):
        X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        c = rng.standard_normal(M).astype(np.complex128)  # real-valued strengths
        g = _cplx(rng, tuple(reversed(nf)), np.complex128)
        gp = _cplx(rng, M, np.complex128)
        fw = _cplx(rng, tuple(reversed(nf)), np.complex128)
        fwr = rng.standard_normal(tuple(reversed(nf))).astype(np.complex128)  # real grid for interp grads
        if dim == 2:
            out_s = sp.spread_2d(*X, c, *nf, kp)
            dx_s = sp.spread_2d_bwd(*nf, kp, (*X, c), g)
            out_i = sp.interp_2d(*X, fw, *nf, kp)
            dx_i = sp.interp_2d_bwd(*nf, kp, (*X, fwr), gp.real.astype(np.complex128))
        else:
            out_s = sp.spread_3d(*X, c, *nf, kp)
            dx_s = sp.spread_3d_bwd(*nf, kp, (*X, c), g)
            out_i = sp.interp_3d(*X, fw, *nf, kp)
            dx_i = sp.interp_3d_bwd(*nf, kp, (*X, fwr), gp.real.astype(np.complex128))
        p = f"d{dim}"
        core[f"{p}/nf"] = np.asarray(nf)
        for d in range(dim):
            core[f"{p}/x{d}"] = X[d]
        core.update({f"{p}/c": c, f"{p}/g": g, f"{p}/gp": gp.real.astype(np.complex128), f"{p}/fw": fw,
                     f"{p}/fwr": fwr, f"{p}/spread": np.asarray(out_s), f"{p}/interp": np.asarray(out_i)})
        for d in range(dim):
            core[f"{p}/spread_bwd_x{d}"] = np.asarray(dx_s[d])
            core[f"{p}/interp_bwd_x{d}"] = np.asarray(dx_i[d])
        core[f"{p}/spread_bwd_c"] = np.asarray(dx_s[dim])
        core[f"{p}/interp_bwd_fw"] = np.asarray(dx_i[dim])
    core["kp"] = np.asarray([kp.nspread, kp.beta, kp.c, kp.upsampfac])
    np.savez_compressed(HERE / "ref_core.npz", **core)


if __name__ == "__main__":
    make(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
