"""GPU test of knn_join_device_noalloc, the join for callers that may not
allocate device memory (applications that own the whole GPU through their own
memory manager, or code that must not allocate once running because
cudaMalloc / cudaFree can block and synchronise the device).

The entry point is called through the C ABI on two different problems in a
row -- the second call runs on scratch the first one left behind -- and each
result must equal knn_join_device's on the same inputs (the same kernels run;
integer data, so the tolerance of the other parity tests is bit-exact).  An
oversize problem must be refused with KNN_EINVAL and a message that states the
bytes it would need.  This file is collected last so that a run stopping at
the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

from knn_sweet_b200 import _lib, data

pytestmark = pytest.mark.gpu


def _join(q, r, k, reps, noalloc, flags=0, **over):
    import torch
    lib = _lib.load()
    m, d = q.shape
    n = r.shape[0]
    idx = torch.full((m, k), -7, dtype=torch.int32, device=q.device)
    dist = torch.full((m, k), -7.0, dtype=torch.float32, device=q.device)
    opt = _lib.default_options()
    opt.qreps = opt.sreps = reps
    opt.flags = flags
    for name, v in over.items():
        setattr(opt, name, v)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [ctypes.c_void_p(q.data_ptr()), m, ctypes.c_void_p(r.data_ptr()), n, d, k,
            ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(dist.data_ptr()),
            ctypes.byref(opt)]
    if noalloc:
        rc = lib.knn_join_device_noalloc(*args, stream)
    else:
        rc = lib.knn_join_device(*args, None, stream)
    torch.cuda.synchronize()
    return rc, idx.cpu().numpy(), dist.cpu().numpy()


def test_noalloc_matches_device_join_two_calls(cuda_device):
    import torch
    big = torch.from_numpy(data.skin_like(data.SKIN_N, seed=1)).to(cuda_device)
    r2 = data.skin_like(20000, seed=77)
    q2 = data.skin_like(3000, seed=78)
    cases = [
        (big, big, 200, 800),  # the full skin self-join, k = 200
        (torch.from_numpy(q2).to(cuda_device), torch.from_numpy(r2).to(cuda_device), 24, 100),
    ]
    for q, r, k, reps in cases:  # two calls in a row on the shared scratch
        rc_ref, i_ref, d_ref = _join(q, r, k, reps, noalloc=False)
        rc, i_got, d_got = _join(q, r, k, reps, noalloc=True)
        assert rc_ref == _lib.KNN_OK
        assert rc == _lib.KNN_OK, _lib.load().knn_last_error()
        assert np.array_equal(i_got, i_ref)
        assert np.array_equal(d_got, d_ref)


def test_noalloc_refuses_oversize(cuda_device):
    import torch
    q = torch.zeros((2_000_000, 3), dtype=torch.float32, device=cuda_device)
    lib = _lib.load()
    # full-size outputs: even a wrongly accepted call stays inside its buffers
    out_i = torch.empty((q.shape[0], 4), dtype=torch.int32, device=cuda_device)
    out_d = torch.empty((q.shape[0], 4), dtype=torch.float32, device=cuda_device)
    rc = lib.knn_join_device_noalloc(ctypes.c_void_p(q.data_ptr()), q.shape[0],
                                     ctypes.c_void_p(q.data_ptr()), q.shape[0], 3, 4,
                                     ctypes.c_void_p(out_i.data_ptr()),
                                     ctypes.c_void_p(out_d.data_ptr()), None, None)
    assert rc == _lib.KNN_EINVAL
    msg = lib.knn_last_error().decode()
    assert "bytes of scratch" in msg and str(32 << 20) in msg


@pytest.mark.parametrize("d,k,n,reps,flags", [
    (32, 16, 30000, 150, 0),                         # tensor-core assignment (d >= 16)
    (64, 10, 20000, 120, 0),                         # generic row width
    (3, 16, 20000, 400, 0),                          # short bands: thread-per-query scan
    (3, 16, 20000, 400, _lib.KNN_SQUARED_DIST),      # squared distances
])
def test_noalloc_matches_device_join_other_shapes(cuda_device, d, k, n, reps, flags):
    """Float data of several widths, the short-band scan and squared distances:
    the same kernels as knn_join_device, so the same result bit for bit, on two
    calls in a row."""
    import torch
    if d == 3:
        r = data.skin_like(n, seed=90 + k) + np.float32(0.25)
        q = r[: n // 5].copy()
    else:
        r, q = data.gaussian_mix(n, 2000, d, 40, seed=91 + d)
    qt, rt = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    for _ in range(2):
        rc_ref, i_ref, d_ref = _join(qt, rt, k, reps, noalloc=False, flags=flags)
        rc, i_got, d_got = _join(qt, rt, k, reps, noalloc=True, flags=flags)
        assert rc_ref == _lib.KNN_OK
        assert rc == _lib.KNN_OK, _lib.load().knn_last_error()
        assert np.array_equal(i_got, i_ref) and np.array_equal(d_got, d_ref)


def test_noalloc_allocates_nothing(cuda_device):
    """After a first call (which looks up the array's device address), further
    calls leave the device's free memory unchanged: no cudaMalloc, no pool."""
    import torch
    lib = _lib.load()
    r = torch.from_numpy(data.skin_like(50000, seed=92)).to(cuda_device)
    m, k = r.shape[0], 32
    idx = torch.empty((m, k), dtype=torch.int32, device=cuda_device)
    dist = torch.empty((m, k), dtype=torch.float32, device=cuda_device)
    opt = _lib.default_options()
    opt.qreps = opt.sreps = 200
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        rc = lib.knn_join_device_noalloc(ctypes.c_void_p(r.data_ptr()), m,
                                         ctypes.c_void_p(r.data_ptr()), m, 3, k,
                                         ctypes.c_void_p(idx.data_ptr()),
                                         ctypes.c_void_p(dist.data_ptr()), ctypes.byref(opt),
                                         stream)
        torch.cuda.synchronize()
        assert rc == _lib.KNN_OK, lib.knn_last_error()
        return idx.cpu().numpy(), dist.cpu().numpy()

    i0, d0 = call()
    free_before = torch.cuda.mem_get_info()[0]
    i1, d1 = call()
    free_after = torch.cuda.mem_get_info()[0]
    assert np.array_equal(i0, i1) and np.array_equal(d0, d1)
    assert free_after == free_before


@pytest.mark.parametrize("what", ["precision", "lloyd_iters"])
def test_noalloc_refuses_options_it_cannot_honour(cuda_device, what):
    import torch
    r = torch.from_numpy(data.skin_like(2000, seed=93)).to(cuda_device)
    over = {"precision": _lib.KNN_BF16_REFINE} if what == "precision" else {"lloyd_iters": 2}
    rc, _, _ = _join(r, r, 8, 20, noalloc=True, **over)
    assert rc == _lib.KNN_EINVAL
    assert what in _lib.load().knn_last_error().decode()
