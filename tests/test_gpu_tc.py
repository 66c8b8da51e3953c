"""Tensor-core (tcgen05, BF16 -> FP32) nearest-representative assignment.

The assignment only has to be approximately nearest (the join recomputes the
exact distance to the chosen representative), so the checks are: an
unambiguous nearest representative is always found; on random data the
chosen representative is within the BF16 rounding bound of the exact nearest;
and whole joins give identical results with and without tensor cores."""
import ctypes

import numpy as np
import pytest

from knn_sweet_b200 import _lib, data, knnjoin

from tests.parity import assert_matches

pytestmark = pytest.mark.gpu


def _assign(points, reps, use_tc):
    import torch
    lib = _lib.load()
    fn = lib.knnsweet_test_assign
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    p = torch.from_numpy(np.ascontiguousarray(points, np.float32)).cuda()
    r = torch.from_numpy(np.ascontiguousarray(reps, np.float32)).cuda()
    n, d = p.shape
    cl = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    dr = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
    rc = fn(p.data_ptr(), n, r.data_ptr(), r.shape[0], d, int(use_tc), cl.data_ptr(),
            dr.data_ptr())
    assert rc == 0, lib.knn_last_error()
    return cl.cpu().numpy(), dr.cpu().numpy()


@pytest.mark.parametrize("d", [16, 32, 40, 128, 256])
def test_unambiguous_nearest_is_found(cuda_device, d):
    rng = np.random.default_rng(d)
    R = 300  # two 256-column tiles, the second partly padding
    reps = rng.uniform(-50, 50, size=(R, d)).astype(np.float32)
    owner = rng.integers(0, R, size=7000)
    pts = reps[owner] + rng.normal(0, 0.05, size=(7000, d)).astype(np.float32)
    cl, dr = _assign(pts, reps, use_tc=True)
    assert np.array_equal(cl, owner)
    exact = np.sqrt(((pts.astype(np.float64) - reps[owner]) ** 2).sum(1))
    np.testing.assert_allclose(dr, exact, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("d", [16, 32, 128])
def test_random_data_within_bf16_bound(cuda_device, d):
    r_, q_ = data.gaussian_mix(20, 9000, d, 40, seed=300 + d)
    pts = q_
    reps = data.gaussian_mix(500, 1, d, 40, seed=400 + d)[0]
    cl_tc, dr_tc = _assign(pts, reps, use_tc=True)
    cl_ex, dr_ex = _assign(pts, reps, use_tc=False)
    assert (cl_tc >= 0).all() and (cl_tc < reps.shape[0]).all()
    # the exact distance to the tensor-core choice is never below the minimum
    assert np.all(dr_tc >= dr_ex * (1 - 1e-6))
    # and exceeds it by at most the BF16 rounding of both vectors
    bound = 2.0 ** -7 * (np.linalg.norm(pts, axis=1) + np.linalg.norm(reps, axis=1).max())
    assert np.all(dr_tc <= dr_ex + bound + 1e-4)
    assert (cl_tc == cl_ex).mean() > 0.9


@pytest.mark.parametrize("d,k", [(32, 32), (128, 16)])
def test_join_identical_with_and_without_tensor_cores(cuda_device, d, k):
    r, q = data.gaussian_mix(30000, 2000, d, 60, seed=500 + d)
    a = knnjoin(q, r, k, qreps=150, sreps=150)
    b = knnjoin(q, r, k, qreps=150, sreps=150, tensor_cores=False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("d,k,iters", [(3, 50, 2), (32, 16, 3)])
def test_lloyd_refinement_keeps_results(cuda_device, oracle, d, k, iters):
    r, q = data.gaussian_mix(25000, 1500, d, 80, seed=600 + d)
    idx, dist, st = knnjoin(q, r, k, qreps=120, sreps=120, lloyd_iters=iters, stats=True)
    oi, od = oracle.bruteforce_f64(q, r, k)
    assert_matches(idx, dist, oi, od)
    b = knnjoin(q, r, k, qreps=120, sreps=120, lloyd_iters=iters)
    assert np.array_equal(idx, b[0]) and np.array_equal(dist, b[1])  # deterministic


@pytest.mark.parametrize("n,d,R", [(5000, 3, 100), (20000, 3, 800), (8000, 32, 300), (3000, 128, 200)])
def test_representative_draw_matches_reference_procedure(cuda_device, oracle, n, d, R):
    """The GPU draw (10 seeded trials scored by pairwise spread) picks the same
    rows as the reference's procedure restated in the oracle."""
    import torch
    if d == 3:
        pts = data.skin_like(n, seed=70 + R)
    else:
        pts = data.gaussian_mix(n, 1, d, 30, seed=71 + d)[0]
    lib = _lib.load()
    fn = lib.knnsweet_test_select_reps
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                   ctypes.c_uint32, ctypes.c_int32, ctypes.c_void_p]
    p = torch.from_numpy(pts).cuda()
    out = torch.full((R,), -1, dtype=torch.int32, device="cuda")
    assert fn(p.data_ptr(), n, d, R, 2015, 10, out.data_ptr()) == 0, lib.knn_last_error()
    want, _ = oracle.select_reps(pts, R, seed=2015, trials=10)
    assert np.array_equal(out.cpu().numpy(), want)
