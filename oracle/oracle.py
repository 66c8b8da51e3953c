"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (knn_oracle.c).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline /
reference arm as the checker.  The product (knn_sweet_b200/) never imports
this module.

Functions
  bruteforce_f64  FP64 brute-force exact kNN (the correctness oracle)
  port_join       the reference's pruned method restated on the CPU
  select_reps     the reference's representative draw (trial spread score)
  glibc_rand_seq  the glibc rand() restatement
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_lib = None


class PortStats(ctypes.Structure):
    _fields_ = [
        ("dist_evals", ctypes.c_int64),
        ("clusters_visited", ctypes.c_int64),
        ("clusters_pruned", ctypes.c_int64),
        ("qreps_trial", ctypes.c_int32),
        ("sreps_trial", ctypes.c_int32),
        ("build_seconds", ctypes.c_double),
        ("scan_seconds", ctypes.c_double),
    ]


def build() -> Path:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        lib = ctypes.CDLL(str(LIB_PATH))
        vp, i64, i32, u32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32
        lib.oracle_bruteforce_f64.argtypes = [vp, i64, vp, i64, i32, i32, vp, i64, vp, vp, ctypes.c_int]
        lib.oracle_bruteforce_f64.restype = ctypes.c_int
        lib.oracle_port_join.argtypes = [vp, i64, vp, i64, i32, i32, i32, i32, u32, i32, vp, i64,
                                         vp, vp, ctypes.POINTER(PortStats), ctypes.c_int]
        lib.oracle_port_join.restype = ctypes.c_int
        lib.oracle_select_reps.argtypes = [vp, i64, i32, i32, u32, i32, vp]
        lib.oracle_select_reps.restype = ctypes.c_int
        lib.oracle_glibc_rand_seq.argtypes = [u32, i64, vp]
        lib.oracle_glibc_rand_seq.restype = None
        lib.oracle_num_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def num_threads() -> int:
    return int(load().oracle_num_threads())


def bruteforce_f64(q, r, k: int, qrows=None, threads: int = 0):
    """FP64 exact kNN: (idx int32 [nq,k], dist float64 [nq,k]); ties -> lower index."""
    q, r = _f32(q), _f32(r)
    m, d = q.shape
    n = r.shape[0]
    rows = None if qrows is None else np.ascontiguousarray(qrows, dtype=np.int64)
    nq = m if rows is None else rows.shape[0]
    idx = np.empty((nq, k), np.int32)
    dist = np.empty((nq, k), np.float64)
    rc = load().oracle_bruteforce_f64(_ptr(q), m, _ptr(r), n, d, k,
                                      None if rows is None else _ptr(rows), nq,
                                      _ptr(idx), _ptr(dist), threads)
    if rc != 0:
        raise ValueError("oracle_bruteforce_f64: bad arguments")
    return idx, dist


def port_join(q, r, k: int, qreps: int, sreps: int, seed: int = 2015, trials: int = 10,
              qrows=None, threads: int = 0):
    """CPU restatement of the reference's pruned join: (idx, dist float32, stats dict)."""
    q, r = _f32(q), _f32(r)
    m, d = q.shape
    n = r.shape[0]
    rows = None if qrows is None else np.ascontiguousarray(qrows, dtype=np.int64)
    nq = m if rows is None else rows.shape[0]
    idx = np.empty((nq, k), np.int32)
    dist = np.empty((nq, k), np.float32)
    st = PortStats()
    rc = load().oracle_port_join(_ptr(q), m, _ptr(r), n, d, k, qreps, sreps, seed, trials,
                                 None if rows is None else _ptr(rows), nq, _ptr(idx), _ptr(dist),
                                 ctypes.byref(st), threads)
    if rc != 0:
        raise ValueError("oracle_port_join: bad arguments")
    stats = {name: getattr(st, name) for name, _ in PortStats._fields_}
    return idx, dist, stats


def select_reps(pts, reps: int, seed: int = 2015, trials: int = 10):
    """Representative rows chosen by the reference's draw: (rows int32 [reps], trial)."""
    pts = _f32(pts)
    n, d = pts.shape
    rows = np.empty(reps, np.int32)
    t = load().oracle_select_reps(_ptr(pts), n, d, reps, seed, trials, _ptr(rows))
    return rows, int(t)


def glibc_rand_seq(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, np.int32)
    load().oracle_glibc_rand_seq(seed, count, _ptr(out))
    return out
