"""CPU tests of the oracle: pinned against the C library's rand(), the golden
known-answer cases and scipy, and the CPU restatement of the reference's
pruned method checked against the FP64 brute force."""
import ctypes
import json
from pathlib import Path

import numpy as np
import pytest

from knn_sweet_b200 import data
from tests.golden.make_golden import cases as golden_cases, load_cases

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_glibc_rand_matches_golden(oracle):
    ref = json.loads((GOLDEN / "glibc_rand.json").read_text())
    for seed, vals in ref.items():
        got = oracle.glibc_rand_seq(int(seed), len(vals))
        assert got.tolist() == vals, seed


def test_glibc_rand_matches_libc_live(oracle):
    libc = ctypes.CDLL("libc.so.6")
    for seed in (2015, 7, 99991):
        libc.srand(ctypes.c_uint(seed))
        want = [libc.rand() for _ in range(5000)]
        assert oracle.glibc_rand_seq(seed, 5000).tolist() == want


def test_golden_fixture_is_current():
    """The committed known answers still describe the committed inputs."""
    live = golden_cases()
    stored = load_cases()
    assert set(live) == set(stored)
    for name, (q, r, k) in live.items():
        sq, sr, sk, _, _ = stored[name]
        assert k == sk and np.array_equal(q, sq) and np.array_equal(r, sr), name


@pytest.mark.parametrize("name", sorted(load_cases()))
def test_bruteforce_matches_golden(oracle, name):
    q, r, k, idx, dist = load_cases()[name]
    gi, gd = oracle.bruteforce_f64(q, r, k)
    assert np.array_equal(gi, idx)
    assert np.array_equal(gd, dist)


def test_golden_tie_rule_by_hand():
    q, r, k, idx, dist = load_cases()["line_d1"]
    # point 5 on a line: itself, then 4 and 6 at distance 1 -> lower index first
    assert idx[5].tolist() == [5, 4, 6]
    assert dist[5].tolist() == [0.0, 1.0, 1.0]
    _, _, _, idx, dist = load_cases()["dups_d3"]
    assert (idx == np.arange(10)).all() and (dist == 0).all()
    _, _, k, idx, dist = load_cases()["k_gt_n"]
    assert (idx[:, 10:] == -1).all() and np.isinf(dist[:, 10:]).all()


@pytest.mark.parametrize("name", sorted(load_cases()))
def test_port_matches_golden(oracle, name):
    q, r, k, idx, dist = load_cases()[name]
    reps = max(1, int(1.6 * np.sqrt(r.shape[0])))
    pi, pd, _ = oracle.port_join(q, r, k, min(reps, q.shape[0]), reps)
    assert np.array_equal(pi, idx)
    np.testing.assert_allclose(pd, dist, rtol=1e-5, atol=0)


@pytest.mark.parametrize("k", [1, 8, 200])
def test_port_exact_on_integer_data(oracle, k):
    x = data.skin_like(12000, seed=3)
    rows = np.arange(0, 12000, 37)
    bi, bd = oracle.bruteforce_f64(x, x, k, qrows=rows)
    pi, pd, st = oracle.port_join(x, x, k, 80, 80, qrows=rows)
    assert np.array_equal(bi, pi)
    assert np.array_equal(bd.astype(np.float32), pd)  # integer data: FP32 exact
    assert st["dist_evals"] < len(rows) * x.shape[0]


def test_port_float_data(oracle):
    r, q = data.gaussian_mix(20000, 1000, 16, 50, seed=5)
    bi, bd = oracle.bruteforce_f64(q, r, 20)
    pi, pd, _ = oracle.port_join(q, r, 20, 60, 120)
    assert (bi == pi).all(axis=1).mean() > 0.999
    np.testing.assert_allclose(pd, bd, rtol=1e-5)


def test_oracle_pinned_to_reference_output(oracle):
    """tests/golden/ref_skin2000_k32.npz holds the reference's own CUDA program's
    full result (2,000 skin-like points joined with themselves, K=32, 50/50
    representatives; made on a B200 by `oracle/compare_ref.py --golden`).  The
    FP64 oracle must reproduce its neighbour distances exactly and its index
    sets up to the order of points tied at the K-th distance (the reference's
    tie order is not deterministic)."""
    z = np.load(GOLDEN / "ref_skin2000_k32.npz")
    x, k = z["x"], int(z["k"])
    ri, rd = z["ref_idx"], z["ref_dist"]
    assert np.array_equal(x, data.skin_like(x.shape[0], seed=int(z["seed"])))
    oi, od = oracle.bruteforce_f64(x, x, k)
    od32 = od.astype(np.float32)
    assert np.array_equal(np.sort(rd, axis=1), od32)
    for i in range(x.shape[0]):
        kth = od32[i, -1]
        assert set(ri[i][rd[i] < kth]) == set(oi[i][od32[i] < kth]), i
        # at the K-th distance both chose the same number of tied points
        assert np.count_nonzero(rd[i] == kth) == np.count_nonzero(od32[i] == kth)


def test_port_matches_reference_output(oracle):
    z = np.load(GOLDEN / "ref_skin2000_k32.npz")
    x, k, reps = z["x"], int(z["k"]), int(z["reps"])
    pi, pd, _ = oracle.port_join(x, x, k, reps, reps)
    assert np.array_equal(np.sort(z["ref_dist"], axis=1), pd)


def test_select_reps_uses_seeded_draw(oracle):
    x = data.skin_like(5000, seed=2)
    rows, trial = oracle.select_reps(x, 50, seed=2015, trials=10)
    draws = oracle.glibc_rand_seq(2015, 500) % 5000
    assert 0 <= trial < 10
    assert rows.tolist() == draws[trial * 50:(trial + 1) * 50].tolist()


def test_data_generators_shapes():
    x = data.skin_like(1000, seed=1)
    assert x.shape == (1000, 3) and x.dtype == np.float32
    assert x.min() >= 0 and x.max() <= 255 and np.all(x == np.rint(x))
    r, q = data.gaussian_mix(500, 50, 32, 10, seed=2)
    assert r.shape == (500, 32) and q.shape == (50, 32)
    pts, off = data.ellipsoid_clouds(8, 256, 512, seed=4)
    assert off[0] == 0 and off[-1] == pts.shape[0] and np.all(np.diff(off) >= 256)
    pairs = data.blob_cloud_pairs(2, 64, 128, seed=5)
    assert len(pairs) == 2 and pairs[0][0].shape[1] == 3
    assert data.skin_like(100, seed=9).tobytes() == data.skin_like(100, seed=9).tobytes()
