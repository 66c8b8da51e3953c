"""ctypes binding of libknnsweet.so (the C ABI declared in include/knnsweet.h).

The library is built in-tree by ``python -m knn_sweet_b200.build``; loading
fails loudly when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libknnsweet.so"

KNN_OK = 0
KNN_EINVAL = -1
KNN_ENOMEM = -2
KNN_ECUDA = -3
KNN_ETIMEOUT = -4
KNN_EINTERNAL = -5
KNN_FP32 = 0
KNN_BF16_REFINE = 1
KNN_SQUARED_DIST = 1
KNN_NO_TENSOR_CORES = 2
KNN_MAX_K = 1024
KNN_MAX_REPS = 8192

# Every function the header declares, with its ctypes signature.
_c_int, _c_i32, _c_i64, _vp = ctypes.c_int, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p


class KnnOptions(ctypes.Structure):
    _fields_ = [
        ("qreps", ctypes.c_int32),
        ("sreps", ctypes.c_int32),
        ("seed", ctypes.c_uint32),
        ("rep_trials", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("margin", ctypes.c_int32),
        ("autotune", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("lloyd_iters", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
    ]


class KnnStats(ctypes.Structure):
    _fields_ = [
        ("dist_evals", ctypes.c_int64),
        ("pairs_total", ctypes.c_int64),
        ("pairs_pruned", ctypes.c_int64),
        ("clusters_visited", ctypes.c_int64),
        ("clusters_pruned", ctypes.c_int64),
        ("fp64_rechecks", ctypes.c_int64),
        ("topk_candidates", ctypes.c_int64),
        ("topk_merges", ctypes.c_int64),
        ("ms_build", ctypes.c_float),
        ("ms_search", ctypes.c_float),
        ("ms_total", ctypes.c_float),
        ("qreps_used", ctypes.c_int32),
        ("sreps_used", ctypes.c_int32),
        ("kernels_launched", ctypes.c_int32),
        ("refine_fallbacks", ctypes.c_int32),
        ("band_queries", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


SIGNATURES = {
    "knn_default_options": (None, [ctypes.POINTER(KnnOptions)]),
    "knn_last_error": (ctypes.c_char_p, []),
    "knn_abi_version": (ctypes.c_int32, []),
    "knn_join": (_c_int, [_vp, _c_i64, _vp, _c_i64, _c_i32, _c_i32, _vp, _vp,
                          ctypes.POINTER(KnnOptions), ctypes.POINTER(KnnStats)]),
    "knn_join_device": (_c_int, [_vp, _c_i64, _vp, _c_i64, _c_i32, _c_i32, _vp, _vp,
                                 ctypes.POINTER(KnnOptions), ctypes.POINTER(KnnStats), _vp]),
    "knn_backward_device": (_c_int, [_vp, _c_i64, _vp, _c_i64, _c_i32, _c_i32, _vp, _vp,
                                     _vp, _vp, _vp]),
    "knn_pack_indexdist": (None, [_vp, _vp, _c_i64, _vp]),
    "knn_trim_memory": (_c_int, []),
    "knn_join_device_noalloc": (_c_int, [_vp, _c_i64, _vp, _c_i64, _c_i32, _c_i32, _vp, _vp,
                                         ctypes.POINTER(KnnOptions), _vp]),
    "knn_index_build": (_c_int, [_vp, _c_i64, _c_i32, ctypes.POINTER(KnnOptions),
                                 ctypes.POINTER(_vp), _vp]),
    "knn_index_query": (_c_int, [_vp, _vp, _c_i64, _c_i32, _vp, _vp,
                                 ctypes.POINTER(KnnOptions), ctypes.POINTER(KnnStats), _vp]),
    "knn_index_free": (_c_int, [_vp]),
    "knn_index_info": (_c_int, [_vp, ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i32),
                                ctypes.POINTER(_c_i32)]),
    "knn_join_batched_device": (_c_int, [_vp, _vp, _vp, _vp, _c_i32, _c_i32, _c_i32, _vp, _vp,
                                         ctypes.POINTER(KnnOptions),
                                         ctypes.POINTER(KnnStats), _vp]),
    "knn_join_partition_device": (_c_int, [_vp, _c_i64, _vp, _c_i64, _c_i32, _c_i32, _c_i32,
                                           _c_i32, _vp, _vp, _vp, ctypes.POINTER(_c_i64),
                                           ctypes.POINTER(KnnOptions),
                                           ctypes.POINTER(KnnStats), _vp]),
    "knn_join_batched": (_c_int, [_vp, _vp, _vp, _vp, _c_i32, _c_i32, _c_i32, _vp, _vp,
                                  ctypes.POINTER(KnnOptions), ctypes.POINTER(KnnStats)]),
    "knn_join_sharded": (_c_int, [_vp, _c_i64, _vp, _c_i64, _c_i32, _c_i32, _vp, _vp,
                                  ctypes.POINTER(KnnOptions), _vp, _c_i32,
                                  ctypes.POINTER(KnnStats)]),
}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


class KnnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"knnsweet error {code}: {msg}")
        self.code = code


def load() -> ctypes.CDLL:
    """Load libknnsweet.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m knn_sweet_b200.build`")
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def check(code: int) -> None:
    if code != KNN_OK:
        msg = load().knn_last_error()
        raise KnnError(code, msg.decode() if msg else "")


def default_options() -> KnnOptions:
    o = KnnOptions()
    load().knn_default_options(ctypes.byref(o))
    return o
