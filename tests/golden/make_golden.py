"""Regenerates the golden fixtures in this folder.

    python tests/golden/make_golden.py

glibc_rand.json  first values of the C library's own rand() after srand(seed)
                 (the generator the reference draws representatives with:
                 src/knnjoin.cu:199-202, 226-229), read through ctypes from
                 libc on the machine that runs this script.
knn_cases.npz    small exact-kNN known-answer cases: hand-made tie-heavy sets
                 plus seeded synthetic sets.  Expected results come from the
                 FP64 brute-force oracle and are cross-checked here against
                 scipy's cKDTree distances before they are written.
"""
from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from knn_sweet_b200 import data  # noqa: E402
from oracle import oracle as O  # noqa: E402

SEEDS = [2015, 1, 0, 12345, 2**31 + 5]


def glibc_fixture():
    libc = ctypes.CDLL("libc.so.6")
    out = {}
    for s in SEEDS:
        libc.srand(ctypes.c_uint(s))
        out[str(s)] = [int(libc.rand()) for _ in range(64)]
    (HERE / "glibc_rand.json").write_text(json.dumps(out, indent=0) + "\n")


def cases():
    rng = np.random.default_rng(20240)
    cs = {}
    line = np.arange(10, dtype=np.float32).reshape(10, 1)
    cs["line_d1"] = (line, line, 3)
    dups = np.tile(np.array([[3.0, 4.0, 5.0]], np.float32), (50, 1))
    cs["dups_d3"] = (dups, dups, 10)
    g = np.stack(np.meshgrid(*[np.arange(6)] * 3, indexing="ij"), -1).reshape(-1, 3)
    g = np.ascontiguousarray(g, dtype=np.float32)
    cs["grid_d3"] = (g, g, 27)
    sk = data.skin_like(800, seed=11)
    cs["skin_d3_k100"] = (sk, sk, 100)
    r, q = data.gaussian_mix(1500, 200, 32, 20, seed=12)
    cs["gauss_d32_k32"] = (q, r, 32)
    small = rng.integers(0, 5, size=(10, 3)).astype(np.float32)
    cs["k_gt_n"] = (small, small, 16)
    d5 = rng.integers(0, 9, size=(400, 5)).astype(np.float32)
    cs["int_d5_k7"] = (d5, d5, 7)
    r40, q40 = data.gaussian_mix(1200, 150, 40, 10, seed=13)
    cs["gauss_d40_k20"] = (q40, r40, 20)
    return cs


def knn_fixture():
    from scipy.spatial import cKDTree

    arrays = {}
    for name, (q, r, k) in cases().items():
        idx, dist = O.bruteforce_f64(q, r, k)
        kk = min(k, r.shape[0])
        dd, _ = cKDTree(r.astype(np.float64)).query(q.astype(np.float64), kk)
        dd = dd.reshape(q.shape[0], kk)
        assert np.allclose(dd, dist[:, :kk], rtol=1e-12, atol=1e-12), name
        arrays[f"{name}__q"] = q
        arrays[f"{name}__r"] = r
        arrays[f"{name}__k"] = np.array(k)
        arrays[f"{name}__idx"] = idx
        arrays[f"{name}__dist"] = dist
    np.savez_compressed(HERE / "knn_cases.npz", **arrays)


def load_cases():
    z = np.load(HERE / "knn_cases.npz")
    names = sorted({key.split("__")[0] for key in z.files})
    return {n: (z[f"{n}__q"], z[f"{n}__r"], int(z[f"{n}__k"]), z[f"{n}__idx"], z[f"{n}__dist"])
            for n in names}


if __name__ == "__main__":
    glibc_fixture()
    knn_fixture()
    print("wrote", HERE / "glibc_rand.json", HERE / "knn_cases.npz")
