"""Reusable index (knn_index_build / knn_index_query): every query batch gives
the result of the one-shot join with the same options, for both forms, and the
index survives the caller's buffer being overwritten."""
import numpy as np
import pytest

from knn_sweet_b200 import data, knnjoin
from knn_sweet_b200.index import KnnIndex

pytestmark = pytest.mark.gpu


def test_queries_match_one_shot_join(cuda_device):
    import torch
    r = torch.from_numpy(data.skin_like(30000, seed=81)).cuda()
    idx = KnnIndex(r, sreps=200)
    assert idx.reps == 200 and idx.n == 30000 and idx.d == 3
    r_copy = r.clone()
    r.fill_(1e6)  # the index keeps its own copy of the points
    for seed in (82, 83):
        q = torch.from_numpy(data.skin_like(7000, seed=seed)).cuda()
        a = idx.query(q, 50, qreps=80)
        b = knnjoin(q, r_copy, 50, qreps=80, sreps=200)
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    idx.free()
    with pytest.raises(RuntimeError):
        idx.query(q, 5)


@pytest.mark.parametrize("d,k,precision", [(32, 32, "fp32"), (32, 32, "bf16_refine"),
                                           (128, 16, "bf16_refine")])
def test_float_data_both_forms(cuda_device, oracle, d, k, precision):
    import torch
    r, q = data.gaussian_mix(25000, 2500, d, 50, seed=90 + d)
    rt, qt = torch.from_numpy(r).cuda(), torch.from_numpy(q).cuda()
    index = KnnIndex(rt, sreps=150, lloyd_iters=2)
    a, ad, st = index.query(qt, k, precision=precision, stats=True, lloyd_iters=2)
    b, bd = knnjoin(qt, rt, k, sreps=150, precision=precision, lloyd_iters=2)
    assert torch.equal(a, b) and torch.equal(ad, bd)
    assert st.sreps_used == 150 and st.dist_evals > 0
    oi, od = oracle.bruteforce_f64(q, r, k)
    np.testing.assert_allclose(ad.cpu().numpy(), od, rtol=1e-5, atol=1e-6)


def test_squared_and_k_above_n(cuda_device):
    import torch
    r = torch.from_numpy(data.gaussian_mix(40, 1, 5, 2, seed=3)[0]).cuda()
    q = torch.from_numpy(data.gaussian_mix(30, 1, 5, 2, seed=4)[0]).cuda()
    index = KnnIndex(r)
    i, d2 = index.query(q, 50, squared=True)
    j, dd = knnjoin(q, r, 50)
    assert torch.equal(i, j)
    assert (i[:, 40:] == -1).all()
    torch.testing.assert_close(d2[:, :40], dd[:, :40] ** 2, rtol=2e-6, atol=0)
