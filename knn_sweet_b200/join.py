"""Python front end of the C ABI (include/knnsweet.h).

The reference's interface is the command line
``knnjoin query_nb source_nb dim qrep_nb srep_nb K query_file source_file``
(src/knnjoin.cu:990-1001) that returns, for every query, K pairs
{source row, Euclidean distance} ascending (src/knnjoin.cu:1104, 1139-1145).
``knnjoin`` below takes the same quantities -- query and source point arrays,
representative counts and K -- and returns the same result as two arrays.

CUDA tensors run on the device through knn_join_device on the current torch
stream; numpy arrays (or CPU tensors) go through knn_join, which copies to the
GPU and back.  Both need libknnsweet.so and a GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

PRECISIONS = {"fp32": _lib.KNN_FP32, "bf16_refine": _lib.KNN_BF16_REFINE}


@dataclass
class JoinStats:
    dist_evals: int
    pairs_total: int
    pairs_pruned: int
    clusters_visited: int
    clusters_pruned: int
    fp64_rechecks: int
    topk_candidates: int
    topk_merges: int
    ms_build: float
    ms_search: float
    ms_total: float
    qreps_used: int
    sreps_used: int
    kernels_launched: int
    refine_fallbacks: int = 0
    band_queries: int = 0


def _options(qreps, sreps, seed, rep_trials, precision, margin,
             squared=False, tensor_cores=True, lloyd_iters=0) -> _lib.KnnOptions:
    o = _lib.default_options()
    o.lloyd_iters = int(lloyd_iters)
    if squared:
        o.flags |= _lib.KNN_SQUARED_DIST
    if not tensor_cores:
        o.flags |= _lib.KNN_NO_TENSOR_CORES
    o.qreps = int(qreps)
    o.sreps = int(sreps)
    o.seed = int(seed) & 0xFFFFFFFF
    o.rep_trials = int(rep_trials)
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    o.precision = PRECISIONS[precision]
    o.margin = int(margin)
    return o


def _is_torch(x) -> bool:
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor)


def knnjoin(queries, sources=None, k: int = 200, *, qreps: int = 0, sreps: int = 0,
            seed: int = 2015, rep_trials: int = 10, precision: str = "fp32",
            margin: int = 32, stats: bool = False, out=None, squared: bool = False,
            tensor_cores: bool = True, lloyd_iters: int = 0):
    """Exact k nearest neighbours of every query row among the source rows.

    queries: (m, d) float32; sources: (n, d) float32 or None for a self-join
    (the reference's sample run joins a set with itself, run_sample.sh:1).
    Returns (idx int32 (m, k), dist float32 (m, k)): per query the k nearest
    by (FP64 squared distance, source row) -- the FP64 brute-force join's set,
    ties to the lower source row -- ascending by FP32 distance; slots beyond n
    hold (-1, inf).  With
    stats=True a JoinStats is returned as a third element.  `out` may give
    preallocated (idx, dist) arrays of the input's kind (e.g. pinned host
    memory for the host path).  squared=True returns squared distances;
    tensor_cores=False keeps every stage on CUDA-core FP32 kernels;
    lloyd_iters > 0 refines the representatives (centroid steps).
    """
    lib = _lib.load()
    opt = _options(qreps, sreps, seed, rep_trials, precision, margin, squared, tensor_cores,
                   lloyd_iters)
    st = _lib.KnnStats()
    stp = ctypes.byref(st) if stats else None
    if _is_torch(queries) and queries.is_cuda:
        import torch
        q = queries.detach()
        if q.dtype != torch.float32 or q.dim() != 2:
            raise ValueError("queries must be a 2-D float32 tensor")
        q = q.contiguous()
        r = q if sources is None else sources.detach().contiguous()
        if r.dtype != torch.float32 or r.dim() != 2 or r.shape[1] != q.shape[1]:
            raise ValueError("sources must be a 2-D float32 tensor with the queries' d")
        if r.device != q.device:
            raise ValueError("queries and sources must be on the same device")
        m, d = q.shape
        n = r.shape[0]
        if out is not None:
            idx, dist = out
            if (idx.shape != (m, k) or dist.shape != (m, k) or idx.dtype != torch.int32
                    or dist.dtype != torch.float32 or not idx.is_contiguous()
                    or not dist.is_contiguous() or idx.device != q.device
                    or dist.device != q.device):
                raise ValueError("out must be contiguous (m, k) int32 / float32 tensors")
        else:
            idx = torch.empty((m, k), dtype=torch.int32, device=q.device)
            dist = torch.empty((m, k), dtype=torch.float32, device=q.device)
        with torch.cuda.device(q.device):
            stream = torch.cuda.current_stream(q.device).cuda_stream
            rc = lib.knn_join_device(
                ctypes.c_void_p(q.data_ptr()), m, ctypes.c_void_p(r.data_ptr()), n, d, k,
                ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(dist.data_ptr()),
                ctypes.byref(opt), stp, ctypes.c_void_p(stream))
        _lib.check(rc)
    else:
        if _is_torch(queries):
            queries = queries.detach().numpy()
        if sources is not None and _is_torch(sources):
            sources = sources.detach().numpy()
        q = np.ascontiguousarray(queries, dtype=np.float32)
        if q.ndim != 2:
            raise ValueError("queries must be 2-D")
        r = q if sources is None else np.ascontiguousarray(sources, dtype=np.float32)
        if r.ndim != 2 or r.shape[1] != q.shape[1]:
            raise ValueError("sources must be 2-D with the queries' d")
        m, d = q.shape
        n = r.shape[0]
        if out is not None:
            idx, dist = out
            if (idx.shape != (m, k) or dist.shape != (m, k) or idx.dtype != np.int32
                    or dist.dtype != np.float32 or not idx.flags.c_contiguous
                    or not dist.flags.c_contiguous):
                raise ValueError("out must be C-contiguous (m, k) int32 / float32 arrays")
        else:
            idx = np.empty((m, k), np.int32)
            dist = np.empty((m, k), np.float32)
        rc = lib.knn_join(q.ctypes.data_as(ctypes.c_void_p), m,
                          r.ctypes.data_as(ctypes.c_void_p), n, d, k,
                          idx.ctypes.data_as(ctypes.c_void_p),
                          dist.ctypes.data_as(ctypes.c_void_p), ctypes.byref(opt), stp)
        _lib.check(rc)
    if stats:
        return idx, dist, JoinStats(**st.as_dict())
    return idx, dist


def knnjoin_sharded(queries, sources=None, k: int = 200, *, devices=(0,), qreps: int = 0,
                    sreps: int = 0, seed: int = 2015, rep_trials: int = 10,
                    precision: str = "fp32", margin: int = 32, stats: bool = False, out=None,
                    squared: bool = False, tensor_cores: bool = True, lloyd_iters: int = 0):
    """knnjoin over several GPUs of this process (knn_join_sharded): the index
    and query clusters are built once on devices[0], the query clusters split
    into len(devices) ranges balanced by estimated work, each device searches
    its range from a peer copy of the index; the result is knnjoin's.  Host
    (numpy) arrays in and out; a device id may repeat."""
    lib = _lib.load()
    opt = _options(qreps, sreps, seed, rep_trials, precision, margin, squared, tensor_cores,
                   lloyd_iters)
    st = _lib.KnnStats()
    q = np.ascontiguousarray(queries, dtype=np.float32)
    if q.ndim != 2:
        raise ValueError("queries must be 2-D")
    r = q if sources is None else np.ascontiguousarray(sources, dtype=np.float32)
    if r.ndim != 2 or r.shape[1] != q.shape[1]:
        raise ValueError("sources must be 2-D with the queries' d")
    m, d = q.shape
    if out is not None:
        idx, dist = out
    else:
        idx = np.empty((m, k), np.int32)
        dist = np.empty((m, k), np.float32)
    dev = np.ascontiguousarray(list(devices), dtype=np.int32)
    rc = lib.knn_join_sharded(q.ctypes.data_as(ctypes.c_void_p), m,
                              r.ctypes.data_as(ctypes.c_void_p), r.shape[0], d, k,
                              idx.ctypes.data_as(ctypes.c_void_p),
                              dist.ctypes.data_as(ctypes.c_void_p), ctypes.byref(opt),
                              dev.ctypes.data_as(ctypes.c_void_p), len(dev),
                              ctypes.byref(st) if stats else None)
    _lib.check(rc)
    if stats:
        return idx, dist, JoinStats(**st.as_dict())
    return idx, dist


def knnjoin_partition(queries, sources=None, k: int = 200, *, part: int, nparts: int,
                      qreps: int = 0, sreps: int = 0, seed: int = 2015, rep_trials: int = 10,
                      precision: str = "fp32", margin: int = 32, stats: bool = False,
                      squared: bool = False, tensor_cores: bool = True, lloyd_iters: int = 0):
    """Part `part` of `nparts` of the join (knn_join_partition_device), for one
    process per GPU: every process passes the same CUDA tensors and options;
    each builds the same index, takes its share of the query clusters and
    returns (idx, dist, rows): full (m, k) tensors in which the rows listed in
    `rows` (int32, this part's queries) hold their results."""
    import torch
    lib = _lib.load()
    opt = _options(qreps, sreps, seed, rep_trials, precision, margin, squared, tensor_cores,
                   lloyd_iters)
    st = _lib.KnnStats()
    q = queries.detach().contiguous()
    r = q if sources is None else sources.detach().contiguous()
    if not q.is_cuda or q.dtype != torch.float32 or q.dim() != 2:
        raise ValueError("queries must be a 2-D float32 CUDA tensor")
    if r.dtype != torch.float32 or r.dim() != 2 or r.shape[1] != q.shape[1] or r.device != q.device:
        raise ValueError("sources must be a 2-D float32 tensor with the queries' d and device")
    m, d = q.shape
    idx = torch.empty((m, k), dtype=torch.int32, device=q.device)
    dist = torch.empty((m, k), dtype=torch.float32, device=q.device)
    rows = torch.empty((m,), dtype=torch.int32, device=q.device)
    count = ctypes.c_int64(0)
    with torch.cuda.device(q.device):
        stream = torch.cuda.current_stream(q.device).cuda_stream
        rc = lib.knn_join_partition_device(
            ctypes.c_void_p(q.data_ptr()), m, ctypes.c_void_p(r.data_ptr()), r.shape[0], d, k,
            int(part), int(nparts), ctypes.c_void_p(idx.data_ptr()),
            ctypes.c_void_p(dist.data_ptr()), ctypes.c_void_p(rows.data_ptr()),
            ctypes.byref(count), ctypes.byref(opt), ctypes.byref(st) if stats else None,
            ctypes.c_void_p(stream))
    _lib.check(rc)
    rows = rows[:count.value]
    if stats:
        return idx, dist, rows, JoinStats(**st.as_dict())
    return idx, dist, rows


def pack_indexdist(idx: np.ndarray, dist: np.ndarray) -> np.ndarray:
    """Interleave into the reference's IndexDist records {int32 index; float dist}."""
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    dist = np.ascontiguousarray(dist, dtype=np.float32)
    out = np.empty(idx.size, dtype=np.dtype([("index", np.int32), ("dist", np.float32)]))
    _lib.load().knn_pack_indexdist(idx.ctypes.data_as(ctypes.c_void_p),
                                   dist.ctypes.data_as(ctypes.c_void_p), idx.size,
                                   out.ctypes.data_as(ctypes.c_void_p))
    return out.reshape(idx.shape)
