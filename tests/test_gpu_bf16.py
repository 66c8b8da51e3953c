"""BF16+refine form (precision="bf16_refine"): tcgen05 distance tiles with
rigorous bounds, exact FP32 re-ranking, FP64 re-check of the k-th boundary.

For d >= 16 the neighbour SET of every query must be the FP64 oracle's
(bit-exact index sets, ties to the lower index); distances are the FP32 ones
of the plain path (within 1e-5 of FP64).  On integer data FP32 is exact, so
the result must equal the plain FP32 join's element for element.  Below
d = 16 the form runs the FP32 scan."""
import numpy as np
import pytest

from knn_sweet_b200 import data, knnjoin

pytestmark = pytest.mark.gpu


def _sets(idx):
    return np.sort(idx, axis=1)


def _int_data(n, d, seed, span=16):
    rng = np.random.default_rng(seed)
    return rng.integers(0, span, size=(n, d)).astype(np.float32)


@pytest.mark.parametrize("d,k", [(16, 50), (32, 200)])
def test_integer_data_identical_to_fp32_and_oracle(cuda_device, oracle, d, k):
    r, q = _int_data(20000, d, seed=d), _int_data(1500, d, seed=d + 1)
    a = knnjoin(q, r, k, qreps=12, sreps=100)
    b, bd, st = knnjoin(q, r, k, qreps=12, sreps=100, precision="bf16_refine", stats=True)
    assert np.array_equal(a[0], b) and np.array_equal(a[1], bd)
    oi, od = oracle.bruteforce_f64(q, r, k)
    assert np.array_equal(b, oi)
    assert st.dist_evals > 0


@pytest.mark.parametrize("d,k", [(16, 32), (32, 32), (40, 20), (128, 100), (200, 16), (256, 8)])
def test_float_data_sets_match_fp64_oracle(cuda_device, oracle, d, k):
    r, q = data.gaussian_mix(20000, 1500, d, 40, seed=700 + d)
    idx, dist, st = knnjoin(q, r, k, sreps=120, precision="bf16_refine", stats=True)
    oi, od = oracle.bruteforce_f64(q, r, k)
    assert np.array_equal(_sets(idx), _sets(oi))
    np.testing.assert_allclose(dist, od, rtol=1e-5, atol=1e-6)
    assert 0 <= st.refine_fallbacks <= q.shape[0]


@pytest.mark.parametrize("d,k", [(1, 10), (3, 50), (8, 16)])
def test_low_dimensions_run_the_fp32_scan(cuda_device, oracle, d, k):
    r, q = data.gaussian_mix(20000, 1500, d, 40, seed=800 + d)
    a = knnjoin(q, r, k, qreps=64, sreps=120)
    b = knnjoin(q, r, k, qreps=64, sreps=120, precision="bf16_refine")
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_large_clusters_many_chunks(cuda_device, oracle):
    # few representatives: every cluster spans many 128-row chunks
    r, q = data.gaussian_mix(40000, 700, 24, 8, seed=77)
    idx, dist = knnjoin(q, r, 64, qreps=4, sreps=6, precision="bf16_refine")
    oi, od = oracle.bruteforce_f64(q, r, 64)
    assert np.array_equal(_sets(idx), _sets(oi))
    np.testing.assert_allclose(dist, od, rtol=1e-5, atol=1e-6)


def test_self_join_with_lloyd_and_squared(cuda_device, oracle):
    pts = data.gaussian_mix(15000, 1, 32, 50, seed=91)[0]
    idx, d2 = knnjoin(pts, k=16, qreps=100, sreps=100, lloyd_iters=2, squared=True,
                      precision="bf16_refine")
    oi, od = oracle.bruteforce_f64(pts, pts, 16)
    assert np.array_equal(_sets(idx), _sets(oi))
    np.testing.assert_allclose(d2, od * od, rtol=2e-5, atol=1e-6)


def test_k_above_n_and_tiny_sets(cuda_device, oracle):
    r, q = data.gaussian_mix(50, 37, 16, 3, seed=5)
    idx, dist = knnjoin(q, r, 64, precision="bf16_refine")
    oi, od = oracle.bruteforce_f64(q, r, 64)
    assert np.array_equal(idx[:, 50:], np.full((37, 14), -1))
    assert np.isinf(dist[:, 50:]).all()
    assert np.array_equal(_sets(idx[:, :50]), _sets(oi[:, :50]))
    one = knnjoin(q[:1], r, 5, precision="bf16_refine")
    assert np.array_equal(_sets(one[0]), _sets(oi[:1, :5]))


def test_duplicates_fall_back_to_scan(cuda_device):
    pts = np.zeros((3000, 16), np.float32)
    pts[1500:] = 1.0
    q = pts[::7].copy()
    idx, dist, st = knnjoin(q, pts, 20, precision="bf16_refine", stats=True)
    ref = knnjoin(q, pts, 20)
    assert np.array_equal(idx, ref[0]) and np.array_equal(dist, ref[1])
    assert st.refine_fallbacks > 0


def test_empty_reference(cuda_device):
    q = np.ones((10, 20), np.float32)
    idx, dist = knnjoin(q, np.zeros((0, 20), np.float32), 3, precision="bf16_refine")
    assert (idx == -1).all() and np.isinf(dist).all()


def test_deterministic(cuda_device):
    r, q = data.gaussian_mix(30000, 2000, 64, 30, seed=12)
    a = knnjoin(q, r, 32, precision="bf16_refine")
    b = knnjoin(q, r, 32, precision="bf16_refine")
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
