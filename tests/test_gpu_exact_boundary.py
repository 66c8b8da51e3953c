"""The k-th boundary of the plain FP32 join is the FP64 join's.

FP32 squared distances rank two points differently from FP64 only inside the
FP32 rounding band of the k-th distance; there the join re-decides the order
in FP64 (in the scan kernel, or in the band kernel for queries whose band did
not fit the scan's candidate list).  These inputs make that band crowded on
purpose: points on the unit sphere (float32-normalised directions) seen from
the centre all lie at distance 1 within a few FP32 units, so their FP32
distances tie in bulk while their FP64 distances differ.  Every top-k variant
is reached: the thread-per-query scan (k <= 32, short bands), the register
list of the warp scan (k <= 24, long bands) and its shared-memory candidate
set (larger k).
"""
import numpy as np
import pytest

from knn_sweet_b200 import knnjoin
from tests.parity import assert_matches

pytestmark = pytest.mark.gpu


def shell_case(n_shell=6000, n_inner=5, seed=0):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n_shell, 3)).astype(np.float32)
    v /= np.linalg.norm(v, axis=1, keepdims=True).astype(np.float32)
    inner = (rng.uniform(-0.3, 0.3, (n_inner, 3))).astype(np.float32)
    r = np.concatenate([v, inner]).astype(np.float32)
    r = r[rng.permutation(r.shape[0])]
    q = np.concatenate([
        np.zeros((4, 3), np.float32),                                  # the centre itself
        rng.uniform(-1e-3, 1e-3, (30, 3)).astype(np.float32),          # near it
        (rng.standard_normal((30, 3)) * 0.5).astype(np.float32),       # anywhere
    ])
    return q, r


@pytest.mark.parametrize("k,sreps", [(8, 0), (16, 0), (32, 0),       # thread scan
                                     (8, 20), (24, 20),               # register list
                                     (32, 20), (64, 20), (200, 20), (1000, 20)])
def test_shell_ties_match_fp64_sets(cuda_device, oracle, k, sreps):
    q, r = shell_case(seed=k)
    idx, dist, st = knnjoin(q, r, k, qreps=4, sreps=sreps, stats=True)
    oi, od = oracle.bruteforce_f64(q, r, k)
    assert_matches(idx, dist, oi, od)
    assert np.all(np.diff(dist, axis=1) >= 0)
    assert st.fp64_rechecks + st.band_queries > 0


@pytest.mark.parametrize("k", [16, 100])
def test_shell_selfjoin_and_squared(cuda_device, oracle, k):
    _, r = shell_case(n_shell=5000, seed=100 + k)
    idx, dist = knnjoin(r, None, k, squared=True)
    oi, od = oracle.bruteforce_f64(r, r, k)
    assert_matches(idx, np.sqrt(dist), oi, od)


def test_band_larger_than_the_band_kernel_buffer(cuda_device, oracle):
    # 20,000 shell points at distance 1 +- a few ulp from the centre: the band
    # kernel's set fills and is cut back many times
    q, r = shell_case(n_shell=20000, n_inner=0, seed=7)
    q = q[:4]
    for k in (1, 300, 1024):
        idx, dist, st = knnjoin(q, r, k, qreps=1, sreps=8, stats=True)
        oi, od = oracle.bruteforce_f64(q, r, k)
        assert_matches(idx, dist, oi, od)
        assert st.band_queries >= 1


def test_integer_ties_unchanged(cuda_device, oracle):
    # small integers: every FP32 squared distance is exact, the join detects it
    # and needs no FP64 step; ties at the k-th keep the lower indices
    rng = np.random.default_rng(3)
    x = rng.integers(0, 6, size=(12000, 3)).astype(np.float32)
    for k in (10, 50, 300):
        idx, dist, st = knnjoin(x, None, k, stats=True)
        rows = np.arange(0, 12000, 61)
        oi, od = oracle.bruteforce_f64(x, x, k, qrows=rows)
        assert_matches(idx[rows], dist[rows], oi, od, exact=True)
        assert st.fp64_rechecks == 0 and st.band_queries == 0


def test_large_integers_take_the_fp64_step(cuda_device, oracle):
    # integers too large for exact FP32 squared distances (2^12 apart in 3-D
    # already exceed 2^24): the FP64 step runs and the sets stay the oracle's
    rng = np.random.default_rng(4)
    r = (rng.integers(0, 3, size=(20000, 3)) * 40000 + rng.integers(0, 9, size=(20000, 3)))
    r = r.astype(np.float32)
    q = r[rng.choice(20000, 300, replace=False)] + 1.0
    idx, dist, st = knnjoin(q, r, 40, stats=True)
    oi, od = oracle.bruteforce_f64(q, r, 40)
    assert_matches(idx, dist, oi, od)
    assert st.fp64_rechecks + st.band_queries > 0
