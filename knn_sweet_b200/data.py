"""Seeded synthetic point sets of the benchmark configurations.

They stand in for the reference's only fixture, the Skin Segmentation table
(4 integer columns in [0,255]; run_sample.sh:1 joins it with itself), and
for the larger workloads the join is measured on.  All generators use
numpy's default_rng(seed) and return C-contiguous float32 arrays.

  skin_like      self-join set: 2-component Gaussian mixture of RGB-like
                 integer points (means (60,80,140) and (180,170,160), sigma 40,
                 weights 0.2075 / 0.7925, clipped to [0,255] and rounded)
  gaussian_mix   reference + query sets from a mixture of isotropic Gaussians
  ellipsoid_clouds  many point clouds on noisy ellipsoid surfaces (CSR)
  blob_cloud_pairs  pairs of clouds of Gaussian blobs in the unit cube
"""
from __future__ import annotations

import numpy as np

SKIN_N = 245_057


def skin_like(n: int = SKIN_N, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    first = rng.random(n) < 0.2075
    means = np.where(first[:, None], np.array([60.0, 80.0, 140.0]),
                     np.array([180.0, 170.0, 160.0]))
    x = means + rng.normal(0.0, 40.0, size=(n, 3))
    return np.ascontiguousarray(np.clip(np.rint(x), 0, 255), dtype=np.float32)


def gaussian_mix(n_ref: int, n_query: int, d: int, centers: int, seed: int,
                 center_kind: str = "uniform", sigma: float = 1.0):
    """(reference, queries) drawn independently from one Gaussian mixture.

    center_kind "uniform": centres uniform in [-10, 10]^d;
    "normal3": centres 3 * N(0, I_d).  Components are chosen uniformly.
    """
    rng = np.random.default_rng(seed)
    if center_kind == "uniform":
        c = rng.uniform(-10.0, 10.0, size=(centers, d))
    elif center_kind == "normal3":
        c = 3.0 * rng.standard_normal(size=(centers, d))
    else:
        raise ValueError(center_kind)
    c = c.astype(np.float32)

    def draw(cnt):
        out = np.empty((cnt, d), np.float32)
        step = 1 << 18
        for s in range(0, cnt, step):
            e = min(cnt, s + step)
            lab = rng.integers(0, centers, size=e - s)
            out[s:e] = c[lab] + np.float32(sigma) * rng.standard_normal(
                size=(e - s, d), dtype=np.float32)
        return out

    ref = draw(n_ref)
    qry = draw(n_query)
    return ref, qry


def config2(scale: float = 1.0):
    """1,000,000 reference / 100,000 query points, d=32, 1,000 centres."""
    return gaussian_mix(int(1_000_000 * scale), int(100_000 * scale), 32, 1000, seed=2)


def config3(scale: float = 1.0):
    """2,000,000 reference / 200,000 query points, d=128, 4,096 centres."""
    return gaussian_mix(int(2_000_000 * scale), int(200_000 * scale), 128, 4096, seed=3,
                        center_kind="normal3", sigma=0.5)


def ellipsoid_clouds(nclouds: int = 4096, lo: int = 256, hi: int = 16384, seed: int = 4,
                     noise: float = 0.01):
    """(points float32 [total, 3], offsets int64 [nclouds + 1])."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=nclouds)
    offsets = np.zeros(nclouds + 1, np.int64)
    np.cumsum(sizes, out=offsets[1:])
    pts = np.empty((int(offsets[-1]), 3), np.float32)
    for c in range(nclouds):
        n = int(sizes[c])
        axes = rng.uniform(0.2, 1.0, size=3)
        v = rng.standard_normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        pts[offsets[c]:offsets[c + 1]] = v * axes + rng.normal(0.0, noise, size=(n, 3))
    return pts, offsets


def blob_cloud_pairs(npairs: int = 64, lo: int = 2048, hi: int = 32768, seed: int = 5,
                     blobs: int = 8, sigma: float = 0.05):
    """List of (x [n1,3], y [n2,3]) float32 pairs in the unit cube."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(npairs):
        pair = []
        for _ in range(2):
            n = int(rng.integers(lo, hi + 1))
            cen = rng.uniform(0.0, 1.0, size=(blobs, 3))
            lab = rng.integers(0, blobs, size=n)
            x = np.clip(cen[lab] + rng.normal(0.0, sigma, size=(n, 3)), 0.0, 1.0)
            pair.append(np.ascontiguousarray(x, dtype=np.float32))
        out.append(tuple(pair))
    return out
