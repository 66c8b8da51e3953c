"""The join over several GPUs (knn_join_sharded, knn_join_partition_device).

knn_join_sharded builds the index and query clusters once on the first listed
device, splits the query clusters into ranges balanced by estimated work and
lets every listed device search its range from a copy of the index, storing
its rows into the first device's result buffer.  knn_join_partition_device
is one such range per process.  The results must be the single join's row for
row, and the FP64 oracle's.  With one GPU the device list repeats device 0:
the shards then run concurrently on their own streams of that device (no
shard waits on another), and the partitions run one after the other.
"""
import numpy as np
import pytest

from knn_sweet_b200 import KnnError, data, knnjoin, knnjoin_partition, knnjoin_sharded
from tests.parity import assert_matches

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("devices", [(0,), (0, 0, 0)])
def test_selfjoin_matches_single_join_and_oracle(cuda_device, oracle, devices):
    x = data.skin_like(30000, seed=21)
    want_i, want_d = knnjoin(x, None, 50, qreps=120, sreps=120)
    idx, dist, st = knnjoin_sharded(x, None, 50, devices=devices, qreps=120, sreps=120,
                                    stats=True)
    assert np.array_equal(idx, want_i) and np.array_equal(dist, want_d)
    rows = np.arange(0, 30000, 29)
    oi, od = oracle.bruteforce_f64(x, x, 50, qrows=rows)
    assert_matches(idx[rows], dist[rows], oi, od, exact=True)
    assert st.pairs_total == 30000 * 30000 and 0 < st.dist_evals < st.pairs_total
    assert st.ms_total > 0 and st.ms_build > 0


@pytest.mark.parametrize("precision", ["fp32", "bf16_refine"])
def test_cross_join_d32_matches_single_join(cuda_device, oracle, precision):
    r, q = data.gaussian_mix(40000, 3001, 32, 40, seed=22)
    want_i, want_d = knnjoin(q, r, 16, qreps=60, sreps=200, precision=precision)
    idx, dist = knnjoin_sharded(q, r, 16, devices=(0, 0), qreps=60, sreps=200,
                                precision=precision)
    assert np.array_equal(idx, want_i) and np.array_equal(dist, want_d)
    oi, od = oracle.bruteforce_f64(q, r, 16)
    assert_matches(idx, dist, oi, od)


def test_fewer_queries_than_shards(cuda_device, oracle):
    r = data.skin_like(5000, seed=23)
    q = r[:2].copy()
    idx, dist = knnjoin_sharded(q, r, 8, devices=(0, 0, 0, 0))
    oi, od = oracle.bruteforce_f64(q, r, 8)
    assert np.array_equal(idx, oi) and np.array_equal(dist, od.astype(np.float32))


def test_bad_device_is_an_error(cuda_device):
    x = data.skin_like(100, seed=24)
    with pytest.raises(KnnError):
        knnjoin_sharded(x, None, 4, devices=(0, 4096))


@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_partitions_cover_the_join(cuda_device, nparts):
    """The parts of knn_join_partition_device are disjoint, cover every query
    and, put together, give the single join's result; they are balanced by
    work (no part gets nothing while another has most)."""
    import torch
    x = data.skin_like(40000, seed=25)
    want_i, want_d = knnjoin(x, None, 64, qreps=200, sreps=200)
    xt = torch.from_numpy(x).cuda()
    got_i = np.full_like(want_i, -7)
    got_d = np.zeros_like(want_d)
    seen = np.zeros(40000, np.int32)
    sizes = []
    for p in range(nparts):
        idx, dist, rows = knnjoin_partition(xt, None, 64, part=p, nparts=nparts, qreps=200,
                                            sreps=200)
        torch.cuda.synchronize()
        rows = rows.cpu().numpy()
        seen[rows] += 1
        got_i[rows] = idx.cpu().numpy()[rows]
        got_d[rows] = dist.cpu().numpy()[rows]
        sizes.append(len(rows))
    assert (seen == 1).all()
    assert np.array_equal(got_i, want_i) and np.array_equal(got_d, want_d)
    if nparts > 1:
        assert min(sizes) > 0.2 * 40000 / nparts
