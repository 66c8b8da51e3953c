"""CPU tests of the C ABI: the library loads, exports every function the
header declares, its structs match the header's layout, and argument errors
come back as status codes without touching a GPU."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from knn_sweet_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(knn_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for want in ("knn_join", "knn_join_device", "knn_last_error", "knn_default_options"):
        assert want in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "knnsweet.h"\n'
        "int main(void){\n"
        'printf("%zu %zu %zu %zu %zu\\n", sizeof(knn_options), sizeof(knn_stats),'
        " offsetof(knn_stats, ms_build), offsetof(knn_stats, qreps_used),"
        " offsetof(knn_options, margin));\n"
        "return 0;}\n")
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    want = [ctypes.sizeof(_lib.KnnOptions), ctypes.sizeof(_lib.KnnStats),
            _lib.KnnStats.ms_build.offset, _lib.KnnStats.qreps_used.offset,
            _lib.KnnOptions.margin.offset]
    assert [int(v) for v in out] == want


def test_default_options():
    o = _lib.default_options()
    assert (o.qreps, o.sreps, o.seed, o.rep_trials, o.precision, o.margin, o.flags) == \
        (0, 0, 2015, 10, _lib.KNN_FP32, 32, 0)
    assert _lib.load().knn_abi_version() == 2


def _call_join(q, r, d, k, opt=None, m=None, n=None):
    lib = _lib.load()
    m = q.shape[0] if m is None else m
    n = r.shape[0] if n is None else n
    idx = np.empty((max(m, 1), max(k, 1)), np.int32)
    dist = np.empty((max(m, 1), max(k, 1)), np.float32)
    return lib.knn_join(q.ctypes.data_as(ctypes.c_void_p), m, r.ctypes.data_as(ctypes.c_void_p), n,
                        d, k, idx.ctypes.data_as(ctypes.c_void_p),
                        dist.ctypes.data_as(ctypes.c_void_p),
                        None if opt is None else ctypes.byref(opt), None)


@pytest.mark.parametrize("d,k", [(0, 5), (-3, 5), (3, 0), (3, -1), (3, 1025)])
def test_bad_sizes_are_rejected(d, k):
    x = np.zeros((4, 3), np.float32)
    assert _call_join(x, x, d, k) == _lib.KNN_EINVAL
    assert _lib.load().knn_last_error()


def test_bad_options_are_rejected():
    x = np.zeros((4, 3), np.float32)
    for field, val in [("flags", 4), ("flags", 0x100), ("qreps", -1), ("sreps", 9000), ("rep_trials", 0),
                       ("precision", 7), ("margin", -2)]:
        o = _lib.default_options()
        setattr(o, field, val)
        assert _call_join(x, x, 3, 2, opt=o) == _lib.KNN_EINVAL, field


def test_empty_query_set_is_ok_without_gpu():
    x = np.zeros((4, 3), np.float32)
    assert _call_join(x, x, 3, 2, m=0) == _lib.KNN_OK


def test_null_pointers_rejected():
    lib = _lib.load()
    out = np.empty((4, 2), np.int32)
    rc = lib.knn_join(None, 4, None, 4, 3, 2, out.ctypes.data_as(ctypes.c_void_p),
                      out.ctypes.data_as(ctypes.c_void_p), None, None)
    assert rc == _lib.KNN_EINVAL
    rc = lib.knn_backward_device(None, 4, None, 4, 3, 2, None, None, None, None, None)
    assert rc == _lib.KNN_EINVAL
    rc = lib.knn_backward_device(None, 4, None, 4, 0, 2, None, None, None, None, None)
    assert rc == _lib.KNN_EINVAL


def test_pack_indexdist_layout():
    from knn_sweet_b200 import pack_indexdist
    idx = np.array([[3, 1], [0, -1]], np.int32)
    dist = np.array([[0.5, 2.0], [0.0, np.inf]], np.float32)
    rec = pack_indexdist(idx, dist)
    raw = rec.view(np.int32).reshape(-1)
    assert raw[0] == 3 and raw[2] == 1 and raw[4] == 0 and raw[6] == -1
    assert rec["dist"][0, 1] == 2.0 and np.isinf(rec["dist"][1, 1])


def _call_batched(qo, ro, ncloud, d, k, opt=None):
    lib = _lib.load()
    qo = np.ascontiguousarray(qo, np.int64)
    ro = np.ascontiguousarray(ro, np.int64)
    return lib.knn_join_batched_device(None, qo.ctypes.data_as(ctypes.c_void_p), None,
                                       ro.ctypes.data_as(ctypes.c_void_p), ncloud, d, k, None,
                                       None, None if opt is None else ctypes.byref(opt), None,
                                       None)


@pytest.mark.parametrize("qo,ro,ncloud,d,k", [
    ([0, 10, 5], [0, 10, 5], 2, 3, 4),      # decreasing offsets
    ([1, 10], [0, 10], 1, 3, 4),            # offsets not starting at 0
    ([0, 10], [0, 10], 1, 0, 4),            # d = 0
    ([0, 10], [0, 10], 1, 33, 4),           # d above the batched limit
    ([0, 10], [0, 10], 1, 3, 257),          # k above the batched limit
    ([0, 10], [0, 10], -1, 3, 4),           # negative cloud count
    ([0, 10], [0, 10], 1, 3, 4),            # null device pointers
])
def test_batched_bad_arguments_rejected(qo, ro, ncloud, d, k):
    assert _call_batched(qo, ro, ncloud, d, k) == _lib.KNN_EINVAL
    assert _lib.load().knn_last_error()


def test_batched_empty_batches_ok_without_gpu():
    assert _call_batched([0], [0], 0, 3, 4) == _lib.KNN_OK
    assert _call_batched([0, 0, 0], [0, 5, 9], 2, 3, 4) == _lib.KNN_OK


def test_batched_bad_options_rejected():
    for field, val in [("flags", 4), ("rep_trials", 0)]:
        o = _lib.default_options()
        setattr(o, field, val)
        assert _call_batched([0, 10], [0, 10], 1, 3, 4, opt=o) == _lib.KNN_EINVAL, field


def test_index_argument_errors_without_gpu():
    lib = _lib.load()
    assert lib.knn_index_free(None) == _lib.KNN_OK
    h = ctypes.c_void_p()
    assert lib.knn_index_build(None, 10, 3, None, ctypes.byref(h), None) == _lib.KNN_EINVAL
    assert lib.knn_index_build(None, 10, 0, None, ctypes.byref(h), None) == _lib.KNN_EINVAL
    assert lib.knn_index_build(None, 10, 3, None, None, None) == _lib.KNN_EINVAL
    assert lib.knn_index_query(None, None, 5, 3, None, None, None, None, None) == _lib.KNN_EINVAL
    assert lib.knn_index_info(None, None, None, None) == _lib.KNN_EINVAL


def test_sharded_argument_errors_without_gpu():
    lib = _lib.load()
    q = np.zeros((4, 3), np.float32)
    idx = np.zeros((4, 2), np.int32)
    dist = np.zeros((4, 2), np.float32)
    dev = np.zeros(2, np.int32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    # no device list, or an empty one
    assert lib.knn_join_sharded(p(q), 4, p(q), 4, 3, 2, p(idx), p(dist), None, None, 2,
                                None) == _lib.KNN_EINVAL
    assert lib.knn_join_sharded(p(q), 4, p(q), 4, 3, 2, p(idx), p(dist), None, p(dev), 0,
                                None) == _lib.KNN_EINVAL
    assert b"device" in lib.knn_last_error()
    # bad sizes come first
    assert lib.knn_join_sharded(p(q), 4, p(q), 4, 3, 0, p(idx), p(dist), None, p(dev), 2,
                                None) == _lib.KNN_EINVAL
    # no queries: nothing to do; no references: every slot empty, as knn_join
    assert lib.knn_join_sharded(None, 0, None, 0, 3, 2, None, None, None, p(dev), 2,
                                None) == _lib.KNN_OK
    assert lib.knn_join_sharded(p(q), 4, None, 0, 3, 2, p(idx), p(dist), None, p(dev), 2,
                                None) == _lib.KNN_OK
    assert (idx == -1).all() and np.isinf(dist).all()


def test_sharded_python_wrapper_errors_without_gpu():
    from knn_sweet_b200 import KnnError, knnjoin_sharded
    x = np.zeros((10, 3), np.float32)
    with pytest.raises(ValueError):
        knnjoin_sharded(np.zeros(10, np.float32), None, 2)
    with pytest.raises(ValueError):
        knnjoin_sharded(x, np.zeros((5, 4), np.float32), 2)
    with pytest.raises(KnnError):
        knnjoin_sharded(x, None, 2, devices=())
    with pytest.raises(KnnError):
        knnjoin_sharded(x, None, 0, devices=(0,))
