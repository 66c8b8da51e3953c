"""Batched join (knn_join_batched_device): many clouds in one call.

Per cloud the result must be what the single join gives for that cloud alone:
checked against the oracle's FP64 brute force per cloud (bit-exact indices on
integer coordinates, where FP32 distances are exact and ties go to the lower
index), against the single-cloud GPU join, and across the CUDA-graph replay.
"""
import numpy as np
import pytest

from knn_sweet_b200 import data, knnjoin
from knn_sweet_b200.batched import BatchedJoinGraph, knnjoin_batched

from tests.parity import assert_sets

pytestmark = pytest.mark.gpu


def _int_clouds(sizes, seed, span=48):
    rng = np.random.default_rng(seed)
    off = np.zeros(len(sizes) + 1, np.int64)
    np.cumsum(sizes, out=off[1:])
    pts = rng.integers(0, span, size=(int(off[-1]), 3)).astype(np.float32)
    return pts, off


def _per_cloud_oracle(oracle, q, qo, r, ro, k):
    idx = np.empty((q.shape[0], k), np.int32)
    dist = np.empty((q.shape[0], k), np.float64)
    for c in range(len(qo) - 1):
        a, b = qo[c], qo[c + 1]
        if a == b:
            continue
        rr = r[ro[c]:ro[c + 1]]
        if rr.shape[0] == 0:
            idx[a:b] = -1
            dist[a:b] = np.inf
            continue
        i, dd = oracle.bruteforce_f64(q[a:b], rr, k)
        idx[a:b], dist[a:b] = i, dd
    return idx, dist


@pytest.mark.parametrize("k", [1, 16, 50])
def test_selfjoin_integer_clouds_bit_exact(cuda_device, oracle, k):
    # sizes: empty, single point, fewer than k, and a spread up to 5000
    sizes = [0, 1, 7, 64, 3000, 0, 250, 5000, 33, 1200, 2]
    pts, off = _int_clouds(sizes, seed=k)
    idx, dist = knnjoin_batched(pts, off, k=k)
    oi, od = _per_cloud_oracle(oracle, pts, off, pts, off, k)
    assert np.array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od.astype(np.float32))


def test_cloud_with_many_representatives(cuda_device, oracle):
    """A cloud of 120,000 points gets 1.6 * sqrt(n) = 554 representatives,
    beyond the 512 that the warp-per-cluster bound kernel takes: that cloud's
    bounds run on the block kernel, the small clouds' in the same call too."""
    sizes = [120_000, 3000, 50]
    pts, off = _int_clouds(sizes, seed=77, span=400)
    k = 8
    idx, dist = knnjoin_batched(pts, off, k=k, autotune=False)
    rows = np.arange(0, sizes[0], 997)
    oi, od = oracle.bruteforce_f64(pts[:sizes[0]], pts[:sizes[0]], k, qrows=rows)
    assert np.array_equal(idx[rows], oi)
    np.testing.assert_array_equal(dist[rows], od.astype(np.float32))
    for c in (1, 2):
        a, b = off[c], off[c + 1]
        oi, od = oracle.bruteforce_f64(pts[a:b], pts[a:b], k)
        assert np.array_equal(idx[a:b], oi)
        np.testing.assert_array_equal(dist[a:b], od.astype(np.float32))


def test_selfjoin_ellipsoid_clouds(cuda_device, oracle):
    pts, off = data.ellipsoid_clouds(nclouds=60, lo=1, hi=4000, seed=11)
    k = 16
    idx, dist = knnjoin_batched(pts, off, k=k)
    oi, od = _per_cloud_oracle(oracle, pts, off, pts, off, k)
    assert_sets(idx, oi)
    np.testing.assert_allclose(dist, od, rtol=2e-6, atol=1e-7)


def test_cross_join_with_empty_sides(cuda_device, oracle):
    pairs = data.blob_cloud_pairs(npairs=12, lo=1, hi=3000, seed=21)
    qs = [p[0] for p in pairs]
    rs = [p[1] for p in pairs]
    qs[3] = qs[3][:0]        # a cloud without queries
    rs[5] = rs[5][:0]        # a cloud without reference points
    rs[7] = rs[7][:4]        # fewer reference points than k
    qo = np.zeros(len(qs) + 1, np.int64)
    ro = np.zeros(len(rs) + 1, np.int64)
    np.cumsum([len(x) for x in qs], out=qo[1:])
    np.cumsum([len(x) for x in rs], out=ro[1:])
    q, r = np.concatenate(qs), np.concatenate(rs)
    k = 10
    idx, dist = knnjoin_batched(q, qo, r, ro, k=k)
    oi, od = _per_cloud_oracle(oracle, q, qo, r, ro, k)
    assert_sets(idx, oi)
    np.testing.assert_allclose(dist, od, rtol=2e-6, atol=1e-7)
    assert (idx[qo[5]:qo[6]] == -1).all() and np.isinf(dist[qo[5]:qo[6]]).all()
    assert (idx[qo[7]:qo[8], 4:] == -1).all()


def test_matches_single_cloud_joins(cuda_device):
    sizes = [900, 17, 4000, 2500]
    pts, off = _int_clouds(sizes, seed=5, span=200)
    idx, dist = knnjoin_batched(pts, off, k=20)
    for c in range(len(sizes)):
        a, b = off[c], off[c + 1]
        si, sd = knnjoin(pts[a:b], k=20)
        assert np.array_equal(idx[a:b], si)
        assert np.array_equal(dist[a:b], sd)


def test_squared_and_device_tensors_and_stats(cuda_device):
    import torch
    pts, off = _int_clouds([300, 2000, 1500], seed=9)
    q = torch.from_numpy(pts).cuda()
    i1, d1, st = knnjoin_batched(q, off, k=8, stats=True)
    i2, d2 = knnjoin_batched(q, torch.from_numpy(off), k=8, squared=True)
    assert torch.equal(i1, i2)
    torch.testing.assert_close(d2, d1 * d1, rtol=1e-6, atol=0)
    sizes = np.diff(off)
    assert st.pairs_total == int((sizes * sizes).sum())
    assert 0 < st.dist_evals < st.pairs_total
    assert st.kernels_launched > 0 and st.ms_total > 0


def test_autotune_does_not_change_results(cuda_device):
    pts, off = _int_clouds([700, 3000, 40, 1800], seed=13)
    a = knnjoin_batched(pts, off, k=12, autotune=True)
    b = knnjoin_batched(pts, off, k=12, autotune=False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_graph_capture_replays_new_points(cuda_device):
    import torch
    sizes = [512, 3000, 1, 900, 2048]
    p1, off = _int_clouds(sizes, seed=31)
    p2, _ = _int_clouds(sizes, seed=32)
    g = BatchedJoinGraph(off, d=3, k=16)
    t1, t2 = torch.from_numpy(p1).cuda(), torch.from_numpy(p2).cuda()
    for p, t in ((p1, t1), (p2, t2), (p1, t1)):
        gi, gd = g(t)
        torch.cuda.synchronize()
        wi, wd = knnjoin_batched(p, off, k=16)
        assert np.array_equal(gi.cpu().numpy(), wi)
        assert np.array_equal(gd.cpu().numpy(), wd)


def test_graph_capture_cross_join(cuda_device):
    import torch
    pairs = data.blob_cloud_pairs(npairs=5, lo=100, hi=2000, seed=41)
    qo = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])]).astype(np.int64)
    ro = np.concatenate([[0], np.cumsum([len(p[1]) for p in pairs])]).astype(np.int64)
    q = torch.from_numpy(np.concatenate([p[0] for p in pairs])).cuda()
    r = torch.from_numpy(np.concatenate([p[1] for p in pairs])).cuda()
    g = BatchedJoinGraph(qo, ro, d=3, k=8)
    gi, gd = g(q, r)
    wi, wd = knnjoin_batched(q, qo, r, ro, k=8)
    torch.cuda.synchronize()
    assert torch.equal(gi, wi) and torch.equal(gd, wd)



def test_host_entry_point_equals_device_entry_point(cuda_device, oracle):
    """knn_join_batched (host buffers, copies inside the call) gives the device
    entry point's result, for a self-join and a cross join."""
    import torch
    pts, off = data.ellipsoid_clouds(nclouds=40, lo=1, hi=3000, seed=31)
    a = knnjoin_batched(pts, off, k=12, autotune=False)
    b = knnjoin_batched(torch.from_numpy(pts).cuda(), off, k=12, autotune=False)
    torch.cuda.synchronize()
    assert np.array_equal(a[0], b[0].cpu().numpy()) and np.array_equal(a[1], b[1].cpu().numpy())
    pairs = data.blob_cloud_pairs(npairs=6, lo=10, hi=2000, seed=32)
    qo = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])]).astype(np.int64)
    ro = np.concatenate([[0], np.cumsum([len(p[1]) for p in pairs])]).astype(np.int64)
    q = np.concatenate([p[0] for p in pairs])
    r = np.concatenate([p[1] for p in pairs])
    hi, hd = knnjoin_batched(q, qo, r, ro, k=5)
    for c in range(len(pairs)):
        oi, od = oracle.bruteforce_f64(q[qo[c]:qo[c + 1]], r[ro[c]:ro[c + 1]], 5)
        assert_sets(hi[qo[c]:qo[c + 1]], oi)
        np.testing.assert_allclose(hd[qo[c]:qo[c + 1]], od, rtol=1e-5, atol=1e-7)
