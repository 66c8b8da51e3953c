"""Batched join: thousands of independent point clouds in one call.

The reference joins one pair of point sets per process run
(src/knnjoin.cu:983-1145).  ``knnjoin_batched`` runs the same exact join for
every cloud of a batch at once through knn_join_batched_device: cloud c's
queries are rows ``q_offsets[c]:q_offsets[c+1]`` and its reference points rows
``r_offsets[c]:r_offsets[c+1]``; neighbours come only from the query's own
cloud and indices are relative to the cloud's first reference row.

``BatchedJoinGraph`` captures the call for fixed offsets in a CUDA graph, so
a training loop that sees the same cloud sizes every step replays one graph
instead of enqueueing the pipeline's launches again.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .join import JoinStats


def _offsets(off, name):
    if off is None:
        return None
    try:
        import torch
        if isinstance(off, torch.Tensor):
            off = off.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    a = np.ascontiguousarray(np.asarray(off, dtype=np.int64))
    if a.ndim != 1 or a.size < 1:
        raise ValueError(f"{name} must be a 1-D array of ncloud + 1 offsets")
    return a


def _batched_options(seed, rep_trials, autotune, squared):
    o = _lib.default_options()
    o.seed = int(seed) & 0xFFFFFFFF
    o.rep_trials = int(rep_trials)
    o.autotune = 1 if autotune else 0
    if squared:
        o.flags |= _lib.KNN_SQUARED_DIST
    return o


def knnjoin_batched(queries, q_offsets, sources=None, r_offsets=None, k: int = 16, *,
                    seed: int = 2015, rep_trials: int = 10, autotune: bool = True,
                    squared: bool = False, stats: bool = False, out=None):
    """k nearest neighbours of every query among its own cloud's points.

    queries: (M, d) float32 CUDA tensor (joined by knn_join_batched_device on
    the current stream) or host array (joined by knn_join_batched, which copies
    in and out itself); q_offsets: ncloud + 1 host offsets.
    sources / r_offsets: the reference clouds, or None for a per-cloud
    self-join.  Returns (idx int32 (M, k), dist float32 (M, k)), indices
    relative to each cloud's first reference row, ascending by distance, ties
    to the lower index, (-1, inf) where a cloud has fewer than k points.
    """
    import torch

    lib = _lib.load()
    qo = _offsets(q_offsets, "q_offsets")
    ro = qo if r_offsets is None else _offsets(r_offsets, "r_offsets")
    if sources is None and r_offsets is not None and not np.array_equal(qo, ro):
        raise ValueError("a self-join takes one set of offsets")
    if qo.size != ro.size:
        raise ValueError("q_offsets and r_offsets must describe the same number of clouds")
    host = not (isinstance(queries, torch.Tensor) and queries.is_cuda)
    if host:
        return _knnjoin_batched_host(lib, queries, qo, sources, ro, k, seed, rep_trials,
                                     autotune, squared, stats, out)
    else:
        q = queries.detach().contiguous()
        r = q if sources is None else sources.detach().contiguous()
    if q.dtype != torch.float32 or q.dim() != 2 or r.dtype != torch.float32 or r.dim() != 2:
        raise ValueError("queries and sources must be 2-D float32")
    if r.shape[1] != q.shape[1] or r.device != q.device:
        raise ValueError("sources must have the queries' d and device")
    M, d = q.shape
    if qo[-1] != M or ro[-1] != r.shape[0]:
        raise ValueError("the last offset must equal the number of rows")
    if out is not None and not host:
        idx, dist = out
        if (idx.shape != (M, k) or dist.shape != (M, k) or idx.dtype != torch.int32
                or dist.dtype != torch.float32 or not idx.is_contiguous()
                or not dist.is_contiguous() or idx.device != q.device or dist.device != q.device):
            raise ValueError("out must be contiguous (M, k) int32 / float32 tensors")
    else:
        idx = torch.empty((M, k), dtype=torch.int32, device=q.device)
        dist = torch.empty((M, k), dtype=torch.float32, device=q.device)
    opt = _batched_options(seed, rep_trials, autotune, squared)
    st = _lib.KnnStats()
    with torch.cuda.device(q.device):
        stream = torch.cuda.current_stream(q.device).cuda_stream
        rc = lib.knn_join_batched_device(
            ctypes.c_void_p(q.data_ptr()), qo.ctypes.data_as(ctypes.c_void_p),
            ctypes.c_void_p(r.data_ptr()), ro.ctypes.data_as(ctypes.c_void_p),
            qo.size - 1, d, k, ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(dist.data_ptr()),
            ctypes.byref(opt), ctypes.byref(st) if stats else None, ctypes.c_void_p(stream))
    _lib.check(rc)
    if host:
        idx, dist = idx.cpu().numpy(), dist.cpu().numpy()
    if stats:
        return idx, dist, JoinStats(**st.as_dict())
    return idx, dist


def _knnjoin_batched_host(lib, queries, qo, sources, ro, k, seed, rep_trials, autotune,
                          squared, stats, out):
    q = np.ascontiguousarray(queries, dtype=np.float32)
    r = q if sources is None else np.ascontiguousarray(sources, dtype=np.float32)
    if q.ndim != 2 or r.ndim != 2 or r.shape[1] != q.shape[1]:
        raise ValueError("queries and sources must be 2-D float32 with the same d")
    M, d = q.shape
    if qo[-1] != M or ro[-1] != r.shape[0]:
        raise ValueError("the last offset must equal the number of rows")
    if out is not None:
        idx, dist = out
        if (idx.shape != (M, k) or dist.shape != (M, k) or idx.dtype != np.int32
                or dist.dtype != np.float32 or not idx.flags.c_contiguous
                or not dist.flags.c_contiguous):
            raise ValueError("out must be C-contiguous (M, k) int32 / float32 arrays")
    else:
        idx = np.empty((M, k), np.int32)
        dist = np.empty((M, k), np.float32)
    opt = _batched_options(seed, rep_trials, autotune, squared)
    st = _lib.KnnStats()
    rc = lib.knn_join_batched(q.ctypes.data_as(ctypes.c_void_p),
                              qo.ctypes.data_as(ctypes.c_void_p),
                              r.ctypes.data_as(ctypes.c_void_p),
                              ro.ctypes.data_as(ctypes.c_void_p), qo.size - 1, d, k,
                              idx.ctypes.data_as(ctypes.c_void_p),
                              dist.ctypes.data_as(ctypes.c_void_p), ctypes.byref(opt),
                              ctypes.byref(st) if stats else None)
    _lib.check(rc)
    if stats:
        return idx, dist, JoinStats(**st.as_dict())
    return idx, dist


class BatchedJoinGraph:
    """The batched join for fixed cloud offsets, captured once in a CUDA graph.

    Construction allocates static input / output buffers on ``device``, runs
    the join once on them (this tunes the representatives per cloud-size
    bucket and warms the allocator) and captures a second call.  Calling the
    object copies new points into the static inputs and replays the graph on
    the current stream; it returns the static (idx, dist) tensors, which the
    next call overwrites.
    """

    def __init__(self, q_offsets, r_offsets=None, *, d: int, k: int = 16, self_join=None,
                 device=None, seed: int = 2015, rep_trials: int = 10, autotune: bool = True,
                 squared: bool = False):
        import torch

        self.q_offsets = _offsets(q_offsets, "q_offsets")
        self.r_offsets = self.q_offsets if r_offsets is None else _offsets(r_offsets, "r_offsets")
        self.self_join = (r_offsets is None) if self_join is None else bool(self_join)
        if self.self_join and not np.array_equal(self.q_offsets, self.r_offsets):
            raise ValueError("a self-join takes one set of offsets")
        self.k = int(k)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        M, N = int(self.q_offsets[-1]), int(self.r_offsets[-1])
        self.q = torch.zeros((M, d), dtype=torch.float32, device=self.device)
        self.r = self.q if self.self_join else torch.zeros((N, d), dtype=torch.float32,
                                                           device=self.device)
        self.idx = torch.empty((M, k), dtype=torch.int32, device=self.device)
        self.dist = torch.empty((M, k), dtype=torch.float32, device=self.device)
        self._kw = dict(seed=seed, rep_trials=rep_trials, autotune=autotune, squared=squared)
        self.graph = None

    def _call(self):
        knnjoin_batched(self.q, self.q_offsets, None if self.self_join else self.r,
                        None if self.self_join else self.r_offsets, self.k,
                        out=(self.idx, self.dist), **self._kw)

    def capture(self, queries, sources=None):
        """Tune and capture on representative data (the clouds' layout, not
        their values, is what the graph fixes)."""
        import torch

        self._load(queries, sources)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self._call()  # tunes (synchronising) and warms the pool
            self._call()
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=side):
            self._call()
        return self

    def _load(self, queries, sources):
        self.q.copy_(queries, non_blocking=True)
        if not self.self_join:
            if sources is None:
                raise ValueError("this graph joins separate reference clouds: pass sources")
            self.r.copy_(sources, non_blocking=True)

    def __call__(self, queries, sources=None):
        if self.graph is None:
            self.capture(queries, sources)
        else:
            self._load(queries, sources)
        self.graph.replay()
        return self.idx, self.dist
