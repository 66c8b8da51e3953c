"""Reusable index of a reference set (knn_index_build / knn_index_query).

The reference recomputes its source-side structures on every run
(clusterReps, src/knnjoin.cu:166-411); ``KnnIndex`` builds them once --
representatives, assignment, distance-sorted member lists -- and joins any
number of query batches against them, each giving the same result as
``knnjoin(queries, sources, k, ...)`` with the same options.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .join import JoinStats, PRECISIONS


class KnnIndex:
    """Index of `sources` ((n, d) float32 CUDA tensor) on its device.

    sreps / seed / rep_trials / lloyd_iters / tensor_cores shape the reference
    clusters as in ``knnjoin``.  The index keeps its own copy of the points."""

    def __init__(self, sources, *, sreps: int = 0, seed: int = 2015, rep_trials: int = 10,
                 lloyd_iters: int = 0, tensor_cores: bool = True):
        import torch
        if not (isinstance(sources, torch.Tensor) and sources.is_cuda):
            raise ValueError("KnnIndex needs a CUDA tensor")
        s = sources.detach()
        if s.dtype != torch.float32 or s.dim() != 2:
            raise ValueError("sources must be a 2-D float32 tensor")
        s = s.contiguous()
        self._lib = _lib.load()
        o = _lib.default_options()
        o.sreps, o.seed, o.rep_trials = int(sreps), int(seed) & 0xFFFFFFFF, int(rep_trials)
        o.lloyd_iters = int(lloyd_iters)
        if not tensor_cores:
            o.flags |= _lib.KNN_NO_TENSOR_CORES
        self.device = s.device
        self.n, self.d = s.shape
        self._h = ctypes.c_void_p()
        with torch.cuda.device(s.device):
            stream = torch.cuda.current_stream(s.device).cuda_stream
            rc = self._lib.knn_index_build(ctypes.c_void_p(s.data_ptr()), self.n, self.d,
                                           ctypes.byref(o), ctypes.byref(self._h),
                                           ctypes.c_void_p(stream))
        _lib.check(rc)
        reps = ctypes.c_int32()
        _lib.check(self._lib.knn_index_info(self._h, None, None, ctypes.byref(reps)))
        self.reps = reps.value

    def query(self, queries, k: int, *, qreps: int = 0, seed: int = 2015, rep_trials: int = 10,
              lloyd_iters: int = 0, precision: str = "fp32", margin: int = 32,
              squared: bool = False, stats: bool = False, out=None):
        """(idx, dist[, JoinStats]) of the k nearest indexed points of every query."""
        import torch
        if self._h is None or not self._h.value:
            raise RuntimeError("the index has been freed")
        q = queries.detach()
        if q.dtype != torch.float32 or q.dim() != 2 or q.shape[1] != self.d:
            raise ValueError("queries must be a 2-D float32 tensor with the index's d")
        if q.device != self.device:
            raise ValueError("queries must be on the index's device")
        q = q.contiguous()
        m = q.shape[0]
        if out is not None:
            idx, dist = out
        else:
            idx = torch.empty((m, k), dtype=torch.int32, device=q.device)
            dist = torch.empty((m, k), dtype=torch.float32, device=q.device)
        o = _lib.default_options()
        o.qreps, o.seed, o.rep_trials = int(qreps), int(seed) & 0xFFFFFFFF, int(rep_trials)
        o.lloyd_iters = int(lloyd_iters)
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        o.precision = PRECISIONS[precision]
        o.margin = int(margin)
        if squared:
            o.flags |= _lib.KNN_SQUARED_DIST
        st = _lib.KnnStats()
        with torch.cuda.device(q.device):
            stream = torch.cuda.current_stream(q.device).cuda_stream
            rc = self._lib.knn_index_query(self._h, ctypes.c_void_p(q.data_ptr()), m, k,
                                           ctypes.c_void_p(idx.data_ptr()),
                                           ctypes.c_void_p(dist.data_ptr()), ctypes.byref(o),
                                           ctypes.byref(st) if stats else None,
                                           ctypes.c_void_p(stream))
        _lib.check(rc)
        if stats:
            return idx, dist, JoinStats(**st.as_dict())
        return idx, dist

    def free(self):
        """Releases the index's device memory (synchronising)."""
        if self._h is not None and self._h.value:
            _lib.check(self._lib.knn_index_free(self._h))
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
