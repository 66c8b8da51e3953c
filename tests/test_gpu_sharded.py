"""knn_join_sharded: the join over several GPUs of one process, by query ranges.

Every shard builds the same reference index and joins its own contiguous range
of queries, so the result must be the single join's, row for row.  With one
GPU the device list repeats device 0: the shards then run concurrently on
their own streams and host threads, the same code path as distinct devices
(nothing in it waits on another shard)."""
import numpy as np
import pytest

from knn_sweet_b200 import KnnError, data, knnjoin, knnjoin_sharded

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("devices", [(0,), (0, 0, 0)])
def test_selfjoin_matches_single_join(cuda_device, devices):
    x = data.skin_like(30000, seed=21)
    want_i, want_d = knnjoin(x, None, 50, qreps=120, sreps=120)
    idx, dist, st = knnjoin_sharded(x, None, 50, devices=devices, qreps=120, sreps=120,
                                    stats=True)
    assert np.array_equal(idx, want_i) and np.array_equal(dist, want_d)
    assert st.pairs_total == 30000 * 30000 and 0 < st.dist_evals < st.pairs_total
    assert st.ms_total > 0


def test_cross_join_d32_matches_single_join(cuda_device):
    r, q = data.gaussian_mix(40000, 3001, 32, 40, seed=22)
    want_i, want_d = knnjoin(q, r, 16, qreps=60, sreps=200)
    idx, dist = knnjoin_sharded(q, r, 16, devices=(0, 0), qreps=60, sreps=200)
    assert np.array_equal(idx, want_i) and np.array_equal(dist, want_d)


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
