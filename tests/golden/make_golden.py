"""Generate the golden fixtures in tests/golden/ (run: python tests/golden/make_golden.py).

The reference (nufftax, pure JAX) cannot be executed here, so the fixtures pin
the oracle to the reference's own test oracles instead:
  * exact FP64 direct sums f[k] = sum_j c_j exp(i isign k.x_j) for types 1/2 and
    f[k] = sum_j c_j exp(i isign s_k.x_j) for type 3, the oracles of
    nufftax tests/conftest.py:154-198 and tests/test_nufft3.py:26-72;
  * the oracle's own outputs on the same seeded inputs (regression values for
    the CUDA path and the oracle);
  * bit-exact bin / cell keys and the stable (bin, cell) permutation for float32
    coordinates that include
    the folding edge cases (x = +-pi, values rounding to the grid end, values
    outside [-pi, pi)).
Inputs are seeded, so the script is reproducible.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import nufft_oracle as O  # noqa: E402


def _c(rng, n, dtype=np.complex128):
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(dtype)


def make_transforms(rng):
    cases = {}
    # (name, dim, M, n_modes, eps, isign)
    specs = [
        ("t1_1d", 1, 500, (64,), [1e-3, 1e-6, 1e-9], 1),
        ("t1_2d", 2, 400, (24, 20), [1e-6], 1),
        ("t1_3d", 3, 300, (10, 12, 8), [1e-6], -1),
    ]
    for name, dim, M, n_modes, epss, isign in specs:
        X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        c = _c(rng, M)
        d = {f"x{i}": X[i] for i in range(dim)}
        d["c"] = c
        d["n_modes"] = np.array(n_modes)
        d["isign"] = np.array(isign)
        d["direct"] = O.direct_type1(X, c, n_modes, isign=isign)
        d["eps"] = np.array(epss)
        for e in epss:
            d[f"oracle_{e:g}"] = O.nufft_type1(X, c, n_modes, eps=e, isign=isign)
        cases[name] = d
    specs2 = [
        ("t2_1d", 1, 500, (64,), [1e-6, 1e-9], -1),
        ("t2_2d", 2, 400, (20, 24), [1e-6], -1),
        ("t2_3d", 3, 300, (8, 12, 10), [1e-6], 1),
    ]
    for name, dim, M, shape, epss, isign in specs2:
        X = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        f = _c(rng, int(np.prod(shape))).reshape(shape)
        vals, flat = O.modes_as_flat(f, dim)
        d = {f"x{i}": X[i] for i in range(dim)}
        d["f"] = f
        d["isign"] = np.array(isign)
        d["direct"] = O.direct_type2(X, vals, flat, isign=isign)
        d["eps"] = np.array(epss)
        for e in epss:
            d[f"oracle_{e:g}"] = O.nufft_type2(X, f, eps=e, isign=isign)
        cases[name] = d
    specs3 = [("t3_1d", 1, 200, 150, 25.0), ("t3_2d", 2, 200, 120, 20.0), ("t3_3d", 3, 150, 100, 8.0)]
    for name, dim, M, K, S in specs3:
        src = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        tgt = [rng.uniform(-S, S, K) for _ in range(dim)]
        c = _c(rng, M)
        eps = 1e-6
        nf = [O.type3_grid_size((a.max() - a.min()) / 2, (b.max() - b.min()) / 2, eps) for a, b in zip(src, tgt)]
        d = {f"x{i}": src[i] for i in range(dim)}
        d.update({f"s{i}": tgt[i] for i in range(dim)})
        d["c"] = c
        d["nf"] = np.array(nf)
        d["direct"] = O.direct_type3(src, c, tgt)
        d["oracle_1e-06"] = O.nufft_type3(src, c, tgt, nf, eps=eps)
        cases[name] = d
    return cases


def make_sort(rng):
    """float32 coordinates with folding edge cases, and their bit-exact bins."""
    cases = {}
    edge = np.array([np.pi, -np.pi, 0.0, np.nextafter(np.float32(np.pi), 0), -np.nextafter(np.float32(np.pi), 0),
                     3.5, -3.5, 7.0, -1e-8, 1e-8, 2.0 * np.pi, -2.0 * np.pi, 1e4, -1e4], dtype=np.float32)
    for dim, nf, tile, ns in ((1, (640,), (64,), 8), (2, (96, 80), (32, 16), 8), (3, (40, 36, 32), (16, 8, 8), 6)):
        M = 3000
        X = [rng.uniform(-np.pi, np.pi, M).astype(np.float32) for _ in range(dim)]
        for i in range(dim):
            X[i][: edge.size] = np.roll(edge, i)
        # a clustered block so some bins hold many points
        for i in range(dim):
            X[i][500:1500] = (0.3 * rng.standard_normal(1000)).astype(np.float32)
        d = {f"x{i}": X[i] for i in range(dim)}
        nbins = int(np.prod([-(-n // t) for n, t in zip(nf, tile)]))
        ncell = int(np.prod(tile))
        for prenorm in (0, 1):
            keys, cells = O.bin_keys(X, nf, ns, tile, bool(prenorm))
            perm, bin_start = O.bin_sort(keys, cells, nbins, ncell)
            d[f"keys_p{prenorm}"] = keys
            d[f"cells_p{prenorm}"] = cells
            d[f"perm_p{prenorm}"] = perm
            d[f"bin_start_p{prenorm}"] = bin_start
        d["nf"] = np.array(nf)
        d["tile"] = np.array(tile)
        d["ns"] = np.array(ns)
        cases[f"sort_{dim}d"] = d
    return cases


def main():
    rng = np.random.default_rng(20261203)
    for name, d in {**make_transforms(rng), **make_sort(rng)}.items():
        np.savez_compressed(HERE / f"{name}.npz", **d)
        print("wrote", name)


if __name__ == "__main__":
    main()
