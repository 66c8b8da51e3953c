"""Differentiation form: loss = sum of the k nearest squared distances in both
directions between two point clouds; forward through the join, backward through
the hand-written kernel.  Checked against FP64 central finite differences of
the loss (h = 1e-4, the join re-run at +-h; coordinates whose neighbour sets
change are skipped) and against a reference gradient (torch autograd of the
gathered squared distances, FP64)."""
import numpy as np
import pytest

from knn_sweet_b200 import data

pytestmark = pytest.mark.gpu


def _clouds(n1=3000, n2=2500, seed=55):
    pairs = data.blob_cloud_pairs(1, lo=min(n1, n2), hi=max(n1, n2), seed=seed)
    return pairs[0]


def _loss64(x, y, k):
    """FP64 loss over the neighbour sets the GPU join picks for (x, y)."""
    import torch
    from knn_sweet_b200 import knnjoin
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    ixy, _ = knnjoin(xt, yt, k)
    iyx, _ = knnjoin(yt, xt, k)
    ixy, iyx = ixy.cpu().numpy(), iyx.cpu().numpy()
    x64, y64 = x.astype(np.float64), y.astype(np.float64)
    l1 = ((x64[:, None, :] - y64[ixy]) ** 2).sum()
    l2 = ((y64[:, None, :] - x64[iyx]) ** 2).sum()
    return l1 + l2, ixy, iyx


@pytest.mark.parametrize("k", [8, 1])
def test_gradient_matches_finite_differences(cuda_device, k):
    import torch
    from knn_sweet_b200.autograd import knn_chamfer
    x, y = _clouds()
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    yt = torch.from_numpy(y).cuda().requires_grad_(True)
    loss = knn_chamfer(xt, yt, k)
    loss.backward()
    gx, gy = xt.grad.cpu().numpy(), yt.grad.cpu().numpy()
    l0, ixy0, iyx0 = _loss64(x, y, k)
    assert abs(float(loss.detach()) - l0) <= 1e-5 * l0

    rng = np.random.default_rng(3)
    h = 1e-4
    checked = 0
    for _ in range(48):
        which = rng.integers(2)
        arr = x if which == 0 else y
        i, c = rng.integers(arr.shape[0]), rng.integers(3)
        vals = []
        same = True
        for sgn in (1.0, -1.0):
            pert = arr.copy()
            pert[i, c] = np.float32(arr[i, c] + sgn * h)
            xs, ys = (pert, y) if which == 0 else (x, pert)
            lv, ixy, iyx = _loss64(xs, ys, k)
            same &= np.array_equal(ixy, ixy0) and np.array_equal(iyx, iyx0)
            vals.append((lv, float(pert[i, c])))
        if not same:
            continue
        (lp, xp), (lm, xm) = vals
        fd = (lp - lm) / (xp - xm)
        g = (gx if which == 0 else gy)[i, c]
        assert abs(g - fd) <= 1e-3 * max(1.0, abs(fd)), (which, i, c, g, fd)
        checked += 1
    assert checked >= 24


def test_gradient_matches_reference_autograd(cuda_device):
    import torch
    from knn_sweet_b200.autograd import knn_dist2
    x, y = _clouds(4000, 6000, seed=56)
    k = 8
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    yt = torch.from_numpy(y).cuda().requires_grad_(True)
    d2, idx = knn_dist2(xt, yt, k)
    w = torch.rand_like(d2)  # arbitrary upstream gradient
    (d2 * w).sum().backward()
    # reference: FP64 autograd of the gathered squared distances, same pairs
    x64 = torch.from_numpy(x).double().cuda().requires_grad_(True)
    y64 = torch.from_numpy(y).double().cuda().requires_grad_(True)
    ref = ((x64.unsqueeze(1) - y64[idx.long()]) ** 2).sum(-1)
    (ref * w.double()).sum().backward()
    assert torch.allclose(d2.double(), ref.detach(), rtol=1e-5, atol=1e-6)
    assert torch.allclose(xt.grad.double(), x64.grad, rtol=1e-4, atol=1e-5)
    assert torch.allclose(yt.grad.double(), y64.grad, rtol=1e-4, atol=1e-5)


def test_self_join_gradient_sums_both_roles(cuda_device):
    import torch
    from knn_sweet_b200.autograd import knn_dist2
    x, _ = _clouds(2048, 2048, seed=57)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    d2, idx = knn_dist2(xt, xt, 4)
    d2.sum().backward()
    x64 = torch.from_numpy(x).double().cuda().requires_grad_(True)
    ((x64.unsqueeze(1) - x64[idx.long()]) ** 2).sum().backward()
    assert torch.allclose(xt.grad.double(), x64.grad, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("k", [1, 8])
def test_batched_chamfer_matches_per_pair(cuda_device, k):
    """The batched differentiable form (one forward call per direction for all
    pairs, one backward launch) gives the per-pair losses' sum and gradients."""
    import torch
    from knn_sweet_b200.autograd import knn_chamfer, knn_chamfer_batched
    pairs = data.blob_cloud_pairs(npairs=6, lo=300, hi=2500, seed=70 + k)
    xs = [torch.from_numpy(p[0]).cuda() for p in pairs]
    ys = [torch.from_numpy(p[1]).cuda() for p in pairs]
    xo = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])]).astype(np.int64)
    yo = np.concatenate([[0], np.cumsum([len(p[1]) for p in pairs])]).astype(np.int64)
    x = torch.cat(xs).requires_grad_(True)
    y = torch.cat(ys).requires_grad_(True)
    loss = knn_chamfer_batched(x, xo, y, yo, k)
    loss.backward()
    ref_loss = 0.0
    gx, gy = [], []
    for a, b in zip(xs, ys):
        a = a.clone().requires_grad_(True)
        b = b.clone().requires_grad_(True)
        l = knn_chamfer(a, b, k)
        l.backward()
        ref_loss += float(l.detach())
        gx.append(a.grad)
        gy.append(b.grad)
    assert float(loss.detach()) == pytest.approx(ref_loss, rel=1e-5)
    # gradients of reference points are sums over every query that picked them,
    # accumulated with float atomics: the order of those additions differs
    # between the two runs
    torch.testing.assert_close(x.grad, torch.cat(gx), rtol=1e-4, atol=1e-5)
    torch.testing.assert_close(y.grad, torch.cat(gy), rtol=1e-4, atol=1e-5)
