"""Every benchmark configuration at full size against the FP64 oracle.

The joins run whole (all queries, all clouds); the oracle checks a seeded
sample: 1,000 queries of the pair joins, 16 whole clouds or cloud pairs of the
batched and differentiation forms.  Bar as everywhere (tests/parity.py): exact
neighbour sets, distances within 1e-5 relative; bit-identical on integer data.
"""
import numpy as np
import pytest

from knn_sweet_b200 import data, knnjoin
from tests.parity import assert_matches, assert_sets

pytestmark = pytest.mark.gpu


def _rows(m, count, seed):
    return np.sort(np.random.default_rng(seed).choice(m, min(m, count), replace=False))


def _device_join(q, r, k, **kw):
    import torch
    qt = torch.from_numpy(q).cuda()
    rt = torch.from_numpy(r).cuda()
    out = knnjoin(qt, rt, k, **kw)
    torch.cuda.synchronize()
    return out[0].cpu().numpy(), out[1].cpu().numpy()


def test_c1_skin_selfjoin_1000_queries(cuda_device, oracle):
    x = data.skin_like(seed=1)
    idx, dist = knnjoin(x, None, 200, qreps=800, sreps=800)
    rows = _rows(x.shape[0], 1000, 101)
    oi, od = oracle.bruteforce_f64(x, x, 200, qrows=rows)
    assert_matches(idx[rows], dist[rows], oi, od, exact=True)


@pytest.mark.parametrize("form", ["fp32", "bf16_refine"])
def test_c2_d32_both_forms(cuda_device, oracle, form):
    r, q = data.config2()
    idx, dist = _device_join(q, r, 32, qreps=1000, sreps=1000, lloyd_iters=3, precision=form)
    rows = _rows(q.shape[0], 1000, 102)
    oi, od = oracle.bruteforce_f64(q, r, 32, qrows=rows)
    assert_matches(idx[rows], dist[rows], oi, od)


@pytest.mark.parametrize("form", ["fp32", "bf16_refine"])
def test_c3_d128_both_forms(cuda_device, oracle, form):
    r, q = data.config3()
    idx, dist = _device_join(q, r, 100, qreps=8192, sreps=8192, lloyd_iters=4, precision=form)
    rows = _rows(q.shape[0], 1000, 103)
    oi, od = oracle.bruteforce_f64(q, r, 100, qrows=rows)
    assert_matches(idx[rows], dist[rows], oi, od)


def test_c4_all_clouds_batched(cuda_device, oracle):
    import torch
    from knn_sweet_b200.batched import BatchedJoinGraph
    pts, off = data.ellipsoid_clouds()
    g = BatchedJoinGraph(off, d=3, k=16)
    idx, dist = g(torch.from_numpy(pts).cuda())
    torch.cuda.synchronize()
    idx, dist = idx.cpu().numpy(), dist.cpu().numpy()
    assert idx.shape == (off[-1], 16) and (idx >= 0).all()
    for c in _rows(len(off) - 1, 16, 104):
        a, b = off[c], off[c + 1]
        oi, od = oracle.bruteforce_f64(pts[a:b], pts[a:b], 16)
        assert_sets(idx[a:b], oi)
        np.testing.assert_allclose(dist[a:b], od, rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("k", [8, 1])
def test_c5_all_pairs_forward_and_gradient(cuda_device, oracle, k):
    import torch
    from knn_sweet_b200.autograd import knn_chamfer_batched, knn_dist2_batched
    pairs = data.blob_cloud_pairs()
    xo = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])]).astype(np.int64)
    yo = np.concatenate([[0], np.cumsum([len(p[1]) for p in pairs])]).astype(np.int64)
    xs = np.concatenate([p[0] for p in pairs])
    ys = np.concatenate([p[1] for p in pairs])
    x = torch.from_numpy(xs).cuda().requires_grad_(True)
    y = torch.from_numpy(ys).cuda().requires_grad_(True)
    knn_chamfer_batched(x, xo, y, yo, k).backward()
    gx, gy = x.grad.double().cpu().numpy(), y.grad.double().cpu().numpy()
    with torch.no_grad():
        dxy, ixy = knn_dist2_batched(x.detach(), xo, y.detach(), yo, k)
        dyx, iyx = knn_dist2_batched(y.detach(), yo, x.detach(), xo, k)
    ixy, iyx, dxy, dyx = (t.cpu().numpy() for t in (ixy, iyx, dxy, dyx))
    for c in _rows(len(pairs), 16, 105):
        xa, xb, ya, yb = xo[c], xo[c + 1], yo[c], yo[c + 1]
        oxy, dxy_o = oracle.bruteforce_f64(xs[xa:xb], ys[ya:yb], k)
        oyx, dyx_o = oracle.bruteforce_f64(ys[ya:yb], xs[xa:xb], k)
        assert_matches(ixy[xa:xb], np.sqrt(dxy[xa:xb]), oxy, dxy_o)
        assert_matches(iyx[ya:yb], np.sqrt(dyx[ya:yb]), oyx, dyx_o)
        # the gradient of the pair's loss equals the FP64 gradient over the
        # oracle's neighbour pairs: the same pairs, so only FP32 rounding
        # differs -- a point's gradient sums dozens of FP32 atomic adds of
        # terms up to the largest component, hence 1e-4 of that component
        px, py = xs[xa:xb].astype(np.float64), ys[ya:yb].astype(np.float64)
        rgx, rgy = np.zeros_like(px), np.zeros_like(py)
        dv = px[:, None, :] - py[oxy]
        rgx += 2 * dv.sum(1)
        np.add.at(rgy, oxy.ravel(), -2 * dv.reshape(-1, 3))
        dv = py[:, None, :] - px[oyx]
        rgy += 2 * dv.sum(1)
        np.add.at(rgx, oyx.ravel(), -2 * dv.reshape(-1, 3))
        scale = max(np.abs(rgx).max(), np.abs(rgy).max())
        assert np.abs(gx[xa:xb] - rgx).max() <= 1e-4 * scale
        assert np.abs(gy[ya:yb] - rgy).max() <= 1e-4 * scale
