"""GPU parity tests of the plain FP32 pruned join against the FP64 oracle.

Bar (tests/parity.py): per query the neighbour index set equals the FP64
join's exactly (ties at equal distance to the lower index), FP32 distances
within 1e-5 relative; on integer data, where every FP32 squared distance is an
exact integer, identical lists and bit-identical distances.
"""
import numpy as np
import pytest

from knn_sweet_b200 import data, knnjoin
from tests.golden.make_golden import load_cases
from tests.parity import assert_matches

pytestmark = pytest.mark.gpu


def torch_join(q, r, k, **kw):
    import torch
    qt = torch.from_numpy(q).cuda()
    rt = qt if r is q else torch.from_numpy(r).cuda()
    out = knnjoin(qt, None if r is q else rt, k, **kw)
    torch.cuda.synchronize()
    return tuple(o.cpu().numpy() if hasattr(o, "cpu") else o for o in out)


@pytest.mark.parametrize("name", sorted(load_cases()))
def test_golden_cases_device_path(cuda_device, name):
    q, r, k, oi, od = load_cases()[name]
    same = np.array_equal(q, r)
    idx, dist = torch_join(q, q if same else r, k)
    exact = bool(np.all(q == np.rint(q)) and np.all(r == np.rint(r)))
    assert_matches(idx, dist, oi, od, exact)


@pytest.mark.parametrize("name", sorted(load_cases()))
def test_golden_cases_host_path(cuda_device, name):
    q, r, k, oi, od = load_cases()[name]
    idx, dist = knnjoin(q, r, k)
    exact = bool(np.all(q == np.rint(q)) and np.all(r == np.rint(r)))
    assert_matches(idx, dist, oi, od, exact)


@pytest.mark.parametrize("k", [1, 16, 100, 200, 256, 257, 600, 1000])
def test_skin_like_selfjoin_k(cuda_device, oracle, k):
    x = data.skin_like(30000, seed=21)
    rows = np.random.default_rng(k).choice(30000, 300, replace=False)
    idx, dist, st = knnjoin(x, None, k, qreps=120, sreps=120, stats=True)
    oi, od = oracle.bruteforce_f64(x, x, k, qrows=rows)
    assert_matches(idx[rows], dist[rows], oi, od, exact=True)
    assert 0 < st.dist_evals <= st.pairs_total
    assert st.pairs_pruned == st.pairs_total - st.dist_evals
    assert np.all(np.diff(dist, axis=1) >= 0)


@pytest.mark.parametrize("d,k", [(1, 5), (2, 9), (5, 7), (8, 32), (16, 64), (32, 32),
                                 (33, 10), (64, 100), (128, 100)])
def test_float_dims(cuda_device, oracle, d, k):
    r, q = data.gaussian_mix(20000, 1000, d, 40, seed=100 + d)
    idx, dist = knnjoin(q, r, k)
    oi, od = oracle.bruteforce_f64(q, r, k)
    assert_matches(idx, dist, oi, od, exact=False)


@pytest.mark.parametrize("k", [129, 200, 256])
def test_float_candidate_set_sorts(cuda_device, oracle, k):
    # k in 129..256: the shared-memory candidate set, compacted by the
    # linear-bin bound of the k-th and sorted at the end by the binned
    # counting sort (float distances: few equal values per bin)
    r, q = data.gaussian_mix(30000, 800, 3, 20, seed=300 + k)
    idx, dist, st = knnjoin(q, r, k, qreps=60, sreps=60, stats=True)
    oi, od = oracle.bruteforce_f64(q, r, k)
    assert_matches(idx, dist, oi, od)
    assert np.all(np.diff(dist, axis=1) >= 0)
    assert st.topk_merges > 0


def test_crowded_bins_take_the_network(cuda_device, oracle):
    # integer points on a small grid: hundreds of candidates share each
    # squared distance, more than a bin of the counting sort takes, so the end
    # of every query sorts by the bitonic network instead
    rng = np.random.default_rng(11)
    x = rng.integers(0, 5, size=(20000, 3)).astype(np.float32)
    rows = np.arange(0, 20000, 97)
    idx, dist = knnjoin(x, None, 200, qreps=30, sreps=30)
    oi, od = oracle.bruteforce_f64(x, x, 200, qrows=rows)
    assert_matches(idx[rows], dist[rows], oi, od, exact=True)


def test_cross_join_separate_reps(cuda_device, oracle):
    r = data.skin_like(25000, seed=31)
    q = data.skin_like(4000, seed=32)
    idx, dist = knnjoin(q, r, 50, qreps=40, sreps=200)
    oi, od = oracle.bruteforce_f64(q, r, 50)
    assert_matches(idx, dist, oi, od, exact=True)


def test_edge_sizes(cuda_device, oracle):
    rng = np.random.default_rng(7)
    for m, n, k in [(1, 1, 1), (1, 5, 8), (7, 3, 4), (3, 300, 300), (50, 50, 50)]:
        q = rng.integers(0, 4, size=(m, 3)).astype(np.float32)
        r = rng.integers(0, 4, size=(n, 3)).astype(np.float32)
        idx, dist = knnjoin(q, r, k)
        oi, od = oracle.bruteforce_f64(q, r, k)
        assert_matches(idx, dist, oi, od, exact=True)


def test_empty_reference_set(cuda_device):
    q = np.ones((4, 3), np.float32)
    r = np.zeros((0, 3), np.float32)
    idx, dist = knnjoin(q, r, 3)
    assert (idx == -1).all() and np.isinf(dist).all()


@pytest.mark.parametrize("k", [64, 200, 600])
def test_all_identical_points(cuda_device, k):
    # every distance equal: the compactions' bound is the common value, the
    # end-of-query sort leaves the binned path (one bin) for the network
    x = np.full((5000, 3), 7.0, np.float32)
    idx, dist = knnjoin(x, None, k)
    assert (dist == 0).all()
    assert (idx == np.arange(k)[None, :]).all()


def test_deterministic_and_apis_agree(cuda_device):
    x = data.skin_like(20000, seed=41)
    a = knnjoin(x, None, 100)
    b = knnjoin(x, None, 100)
    c = torch_join(x, x, 100)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    for u, v in zip(a, c):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("m,k", [(60000, 40), (33333, 200), (100000, 200)])
def test_host_path_chunked_copies_match_device_path(cuda_device, m, k):
    """Large host-buffer joins scan in row chunks (about 16 MB of results each,
    8 to 32 chunks: 160 MB here gives 9) and copy each chunk back while the
    next runs; the result must equal the device-buffer join's."""
    x = data.skin_like(m, seed=61)
    a = knnjoin(x, None, k)
    b = torch_join(x, x, k)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    r, q = data.gaussian_mix(50000, m, 8, 30, seed=62)
    c = knnjoin(q, r, k, qreps=300, sreps=300)
    e = torch_join(q, r, k, qreps=300, sreps=300)
    for u, v in zip(c, e):
        assert np.array_equal(u, v)


def test_rep_counts_do_not_change_result(cuda_device):
    x = data.skin_like(15000, seed=51)
    base = knnjoin(x, None, 32, qreps=1, sreps=1)
    for reps in (7, 64, 500, 4096):
        got = knnjoin(x, None, 32, qreps=reps, sreps=reps)
        assert np.array_equal(base[0], got[0]) and np.array_equal(base[1], got[1])


def test_matches_reference_program_output(cuda_device):
    """Against the reference's own CUDA program's result on the same points
    (tests/golden/ref_skin2000_k32.npz): identical sorted distances, identical
    index sets below the K-th distance, the same number of points at it."""
    from pathlib import Path
    z = np.load(Path(__file__).resolve().parent / "golden" / "ref_skin2000_k32.npz")
    x, k, reps = z["x"], int(z["k"]), int(z["reps"])
    idx, dist = knnjoin(x, None, k, qreps=reps, sreps=reps)
    ri, rd = z["ref_idx"], z["ref_dist"]
    assert np.array_equal(dist, np.sort(rd, axis=1))
    for i in range(x.shape[0]):
        kth = dist[i, -1]
        assert set(idx[i][dist[i] < kth]) == set(ri[i][rd[i] < kth])


def test_full_size_skin_selfjoin_properties(cuda_device, oracle):
    """The full self-join workload (245,057 points, k=200, 800/800 reps):
    size-independent properties on all rows, oracle comparison on a sample."""
    x = data.skin_like(seed=1)
    idx, dist, st = knnjoin(x, None, 200, qreps=800, sreps=800, stats=True)
    n = x.shape[0]
    assert idx.shape == (n, 200)
    assert np.all(np.diff(dist, axis=1) >= 0)
    assert (idx >= 0).all() and (idx < n).all()
    assert (dist[:, 0] == 0).all()
    # no duplicate neighbour in a row
    s = np.sort(idx, axis=1)
    assert not np.any(s[:, 1:] == s[:, :-1])
    rows = np.random.default_rng(3).choice(n, 256, replace=False)
    oi, od = oracle.bruteforce_f64(x, x, 200, qrows=rows)
    assert_matches(idx[rows], dist[rows], oi, od, exact=True)
    assert st.dist_evals < 0.05 * st.pairs_total


def test_host_calls_from_several_threads(cuda_device):
    """Host-buffer joins keep two streams per calling thread: joins issued from
    several threads at once (each with its own chunked copy-back) return what
    the same joins return one at a time."""
    import threading
    xs = [data.skin_like(40000, seed=70 + i) for i in range(4)]
    want = [knnjoin(x, None, 64) for x in xs]
    got = [None] * len(xs)
    errors = []

    def run(i):
        try:
            for _ in range(3):
                got[i] = knnjoin(xs[i], None, 64)
        except Exception as e:  # reported below
            errors.append(e)
    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(xs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for w, g in zip(want, got):
        assert np.array_equal(w[0], g[0]) and np.array_equal(w[1], g[1])
