"""Parity checks against the FP64 brute-force oracle, shared by the GPU tests.

The bar, for every form of the join:
  - per query, the neighbour index SET equals the FP64 join's (the k nearest by
    (FP64 squared distance, index): ties at equal distance go to the lower
    index), exactly;
  - distances within 1e-5 relative of the oracle's, position by position (the
    library lists a query's neighbours by FP32 distance, the oracle by FP64;
    sorted lists of values each within the tolerance stay within it);
  - on integer data every FP32 squared distance is an exact integer, so there
    the lists themselves and the distances are bit-identical (exact=True).
"""
from __future__ import annotations

import numpy as np

REL = 1e-5


def assert_sets(idx, oi) -> None:
    idx = np.asarray(idx)
    oi = np.asarray(oi)
    assert idx.shape == oi.shape, (idx.shape, oi.shape)
    a, b = np.sort(idx, axis=1), np.sort(oi, axis=1)
    bad = np.flatnonzero((a != b).any(axis=1))
    assert bad.size == 0, (
        f"{bad.size} of {idx.shape[0]} queries differ from the FP64 oracle's neighbour set; "
        f"first: row {bad[0]}: extra {sorted(set(a[bad[0]]) - set(b[bad[0]]))}, "
        f"missing {sorted(set(b[bad[0]]) - set(a[bad[0]]))}")


def assert_dists(dist, od, rel: float = REL) -> None:
    dist = np.asarray(dist)
    fin = np.isfinite(od)
    assert np.array_equal(np.isfinite(dist), fin)
    np.testing.assert_allclose(dist[fin], od[fin], rtol=rel, atol=0)


def assert_matches(idx, dist, oi, od, exact: bool = False) -> None:
    idx = np.asarray(idx)
    dist = np.asarray(dist)
    if exact:
        assert np.array_equal(idx, oi)
        assert np.array_equal(dist, od.astype(np.float32))
        return
    assert_sets(idx, oi)
    assert_dists(dist, od)
