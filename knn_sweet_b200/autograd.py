"""Differentiable kNN squared distances over the C ABI.

``knn_dist2(queries, sources, k)`` returns, for every query row, its k nearest
source rows (``idx``) and the squared distances ``d2[i, t] = |q_i - s_idx|^2``
as a tensor that is differentiable with respect to both point sets.  The
neighbour sets are constants of the forward pass (the join is piecewise
constant in the coordinates); the backward pass is the hand-written kernel
``knn_backward_device`` (csrc/backward.cu):

    grad_q[i] += 2 g (q_i - s_j),      grad_s[j] -= 2 g (q_i - s_j).

The reference computes no gradient; this is the "differentiation form" of
the join (e.g. kNN Chamfer losses between point clouds).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .join import knnjoin


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


class _KnnDist2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, queries, sources, k, qreps, sreps):
        q = queries.detach().contiguous()
        s = sources.detach().contiguous()
        # the join writes the squared distances it ranked by (FP32, summed in
        # dimension order); missing neighbours are (-1, +inf)
        idx, d2 = knnjoin(q, s, k, qreps=qreps, sreps=sreps, squared=True)
        ctx.save_for_backward(q, s, idx)
        ctx.mark_non_differentiable(idx)
        return d2, idx

    @staticmethod
    def backward(ctx, grad_d2, _grad_idx):
        q, s, idx = ctx.saved_tensors
        m, d = q.shape
        n = s.shape[0]
        k = idx.shape[1]
        g = grad_d2.contiguous().to(torch.float32)
        g = torch.where(idx >= 0, g, torch.zeros_like(g))
        grad_q = torch.zeros_like(q)
        grad_s = torch.zeros_like(s) if ctx.needs_input_grad[1] else None
        lib = _lib.load()
        with torch.cuda.device(q.device):
            stream = ctypes.c_void_p(torch.cuda.current_stream(q.device).cuda_stream)
            rc = lib.knn_backward_device(_ptr(q), m, _ptr(s), n, d, k, _ptr(idx), _ptr(g),
                                         _ptr(grad_q),
                                         _ptr(grad_s) if grad_s is not None else None, stream)
        _lib.check(rc)
        return grad_q, grad_s, None, None, None


def knn_dist2(queries: torch.Tensor, sources: torch.Tensor, k: int, *, qreps: int = 0,
              sreps: int = 0):
    """(d2, idx): k nearest squared distances (differentiable) and indices."""
    if not (queries.is_cuda and sources.is_cuda):
        raise ValueError("knn_dist2 needs CUDA tensors")
    return _KnnDist2.apply(queries, sources, k, qreps, sreps)


def knn_chamfer(x: torch.Tensor, y: torch.Tensor, k: int = 1) -> torch.Tensor:
    """Sum of the k nearest squared distances in both directions:
    sum_i sum_t |x_i - y_nn(i,t)|^2 + sum_j sum_t |y_j - x_nn(j,t)|^2
    (k = 1 is the Chamfer distance)."""
    dxy, _ = knn_dist2(x, y, k)
    dyx, _ = knn_dist2(y, x, k)
    return dxy.sum() + dyx.sum()


def _cloud_base(offsets, rows_off, device):
    """Per query row: the first row of its cloud's reference points.  Built on
    the device from the per-cloud values (a host-side expansion meant a
    row-sized pageable copy on every forward pass)."""
    import numpy as np
    qo = np.asarray(rows_off, dtype=np.int64)
    ro = np.asarray(offsets, dtype=np.int64)
    base = torch.as_tensor(ro[:-1].astype(np.int32)).to(device, non_blocking=True)
    counts = torch.as_tensor(np.diff(qo)).to(device, non_blocking=True)
    return torch.repeat_interleave(base, counts, output_size=int(qo[-1]))


class _KnnDist2Batched(torch.autograd.Function):
    @staticmethod
    def forward(ctx, queries, q_offsets, sources, r_offsets, k):
        from .batched import knnjoin_batched
        q = queries.detach().contiguous()
        s = sources.detach().contiguous()
        idx, d2 = knnjoin_batched(q, q_offsets, s, r_offsets, k, squared=True)
        # indices relative to each cloud -> rows of the concatenated sources
        base = _cloud_base(r_offsets, q_offsets, q.device)
        gidx = torch.where(idx >= 0, idx + base[:, None], idx)
        ctx.save_for_backward(q, s, gidx)
        ctx.mark_non_differentiable(idx)
        return d2, idx

    @staticmethod
    def backward(ctx, grad_d2, _grad_idx):
        q, s, gidx = ctx.saved_tensors
        m, d = q.shape
        n, k = s.shape[0], gidx.shape[1]
        g = torch.where(gidx >= 0, grad_d2.contiguous().to(torch.float32),
                        torch.zeros_like(grad_d2, dtype=torch.float32))
        grad_q = torch.zeros_like(q)
        grad_s = torch.zeros_like(s) if ctx.needs_input_grad[2] else None
        lib = _lib.load()
        with torch.cuda.device(q.device):
            stream = ctypes.c_void_p(torch.cuda.current_stream(q.device).cuda_stream)
            rc = lib.knn_backward_device(_ptr(q), m, _ptr(s), n, d, k, _ptr(gidx), _ptr(g),
                                         _ptr(grad_q),
                                         _ptr(grad_s) if grad_s is not None else None, stream)
        _lib.check(rc)
        return grad_q, None, grad_s, None, None


def knn_dist2_batched(queries, q_offsets, sources, r_offsets, k: int):
    """Batched (d2, idx) over many cloud pairs: cloud c's queries
    q_offsets[c]:q_offsets[c+1] against its sources r_offsets[c]:r_offsets[c+1];
    idx relative to the cloud's first source row; d2 differentiable in both point
    sets (one forward call for all clouds, one backward launch)."""
    if not (queries.is_cuda and sources.is_cuda):
        raise ValueError("knn_dist2_batched needs CUDA tensors")
    return _KnnDist2Batched.apply(queries, q_offsets, sources, r_offsets, k)


def knn_chamfer_batched(x, x_offsets, y, y_offsets, k: int = 1) -> torch.Tensor:
    """Per-pair Chamfer-type losses of many cloud pairs, summed: for every pair c,
    the k nearest squared distances from x_c to y_c and from y_c to x_c."""
    dxy, _ = knn_dist2_batched(x, x_offsets, y, y_offsets, k)
    dyx, _ = knn_dist2_batched(y, y_offsets, x, x_offsets, k)
    return dxy.sum() + dyx.sum()
