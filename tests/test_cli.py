"""The `knnjoin` command line: the reference's argv, inputs and output lines
(src/knnjoin.cu:983-1172, include/common8.h:92-135).  Input parsing is checked
on the CPU (KNNJOIN_DUMP_INPUT stops before the join); the join itself on the
GPU against the FP64 oracle."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from knn_sweet_b200 import data

ROOT = Path(__file__).resolve().parent.parent
CLI = ROOT / "knn_sweet_b200" / "bin" / "knnjoin"
# the reference's fixture, where a checkout of the reference is named by
# KNN_REFERENCE_ROOT (the test is skipped otherwise)
_REF_ROOT = os.environ.get("KNN_REFERENCE_ROOT")
SKIN = Path(_REF_ROOT, "test", "Skin_NonSkin.txt") if _REF_ROOT else None


def run_cli(args, env_extra=None, check=True):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True,
                          env=env, check=check)


def dumped_inputs(path, m, n, d):
    raw = np.fromfile(path, dtype=np.float32)
    assert raw.size == (m + n) * d
    return raw[:m * d].reshape(m, d), raw[m * d:].reshape(n, d)


def reference_random(m, n, d, oracle):
    """pointSetup's "random" mode: after srand(2015) every value is
    rand()%10 + (float)rand()/RAND_MAX, left call first, queries then sources."""
    r = oracle.glibc_rand_seq(2015, 2 * (m + n) * d).astype(np.int64)
    a, b = r[0::2], r[1::2]
    vals = (a % 10).astype(np.float32) + b.astype(np.float32) / np.float32(2147483647)
    return vals[:m * d].reshape(m, d), vals[m * d:].reshape(n, d)


def test_usage_without_arguments():
    res = run_cli([], check=False)
    assert res.returncode == 1 and "usage" in res.stdout


def test_random_inputs_match_reference_generator(tmp_path, oracle):
    out = tmp_path / "in.bin"
    res = run_cli([50, 70, 3, 4, 4, 5, "random", "random"], {"KNNJOIN_DUMP_INPUT": str(out)})
    assert "query data random" in res.stdout and "source data random" in res.stdout
    q, r = dumped_inputs(out, 50, 70, 3)
    wq, wr = reference_random(50, 70, 3, oracle)
    assert np.array_equal(q, wq) and np.array_equal(r, wr)


def test_text_reader_crlf_and_token_stream(tmp_path):
    x = data.skin_like(300, seed=5)
    lab = (np.arange(300) % 2 + 1).astype(np.float32)
    rows = np.column_stack([x, lab])  # 4 columns like the skin table
    f = tmp_path / "pts.txt"
    f.write_bytes("".join("\t".join(str(int(v)) for v in row) + "\r\n" for row in rows).encode())
    out = tmp_path / "in.bin"
    # dim 4: whole rows
    run_cli([300, 250, 4, 8, 8, 5, f, f], {"KNNJOIN_DUMP_INPUT": str(out)})
    q, r = dumped_inputs(out, 300, 250, 4)
    assert np.array_equal(q, rows) and np.array_equal(r, rows[:250])
    # dim 3 over 4-column rows: the reference reads a plain token stream
    run_cli([200, 100, 3, 8, 8, 5, f, f], {"KNNJOIN_DUMP_INPUT": str(out)})
    q, r = dumped_inputs(out, 200, 100, 3)
    stream = rows.reshape(-1)
    assert np.array_equal(q.reshape(-1), stream[:600])
    assert np.array_equal(r.reshape(-1), stream[:300])


def _float_text(vals, rng):
    """float32 values as text in mixed spellings and separators."""
    seps = [" ", "\t", "\n", "\r\n", "  \t "]
    parts = []
    for i, v in enumerate(vals):
        form = ("%.9g", "%.8e", "%.9G")[i % 3]
        parts.append(form % float(v))
        parts.append(seps[rng.integers(len(seps))])
    return "".join(parts)


def test_parallel_text_reader_equals_serial_reading(tmp_path):
    rng = np.random.default_rng(11)
    vals = (rng.standard_normal(120_000) * 10.0 ** rng.integers(-6, 7, 120_000)).astype(np.float32)
    f = tmp_path / "big.txt"
    f.write_text(_float_text(vals, rng))
    assert f.stat().st_size > 16 * (1 << 16)  # many chunks
    out = tmp_path / "in.bin"
    run_cli([40_000, 30_000, 3, 8, 8, 5, f, f],
            {"KNNJOIN_DUMP_INPUT": str(out), "OMP_NUM_THREADS": "4"})
    q, r = dumped_inputs(out, 40_000, 30_000, 3)
    assert np.array_equal(q.reshape(-1), vals) and np.array_equal(r.reshape(-1), vals[:90_000])


def test_parallel_text_reader_stops_like_fscanf(tmp_path):
    """Text that is not a whole number deep in the file: "1.5-2" reads as two
    values, "7abc" as 7 followed by the end of the input, as successive
    fscanf("%f") calls read them; the slots past the end stay zero."""
    rng = np.random.default_rng(12)
    a = rng.standard_normal(60_000).astype(np.float32)
    b = rng.standard_normal(30_000).astype(np.float32)
    c = rng.standard_normal(20_000).astype(np.float32)
    f = tmp_path / "odd.txt"
    f.write_text(_float_text(a, rng) + " 1.5-2 " + _float_text(b, rng) + " 7abc "
                 + _float_text(c, rng))
    want = np.concatenate([a, [1.5, -2.0], b, [7.0]]).astype(np.float32)
    m = want.size + 50
    out = tmp_path / "in.bin"
    res = run_cli([m, 1000, 1, 8, 8, 5, f, f],
                  {"KNNJOIN_DUMP_INPUT": str(out), "OMP_NUM_THREADS": "4"})
    assert "error reading" in res.stdout
    q, r = dumped_inputs(out, m, 1000, 1)
    assert np.array_equal(q[:want.size, 0], want) and not q[want.size:].any()
    assert np.array_equal(r[:, 0], a[:1000])


def test_raw_float32_inputs(tmp_path):
    rng = np.random.default_rng(13)
    x = rng.standard_normal((500, 4)).astype(np.float32)
    f = tmp_path / "pts.f32"
    x.tofile(f)
    out = tmp_path / "in.bin"
    run_cli([500, 300, 4, 8, 8, 5, f, f], {"KNNJOIN_DUMP_INPUT": str(out)})
    q, r = dumped_inputs(out, 500, 300, 4)
    assert np.array_equal(q, x) and np.array_equal(r, x[:300])


def test_missing_file_is_an_error(tmp_path):
    res = run_cli([5, 5, 3, 2, 2, 2, tmp_path / "nope.txt", tmp_path / "nope.txt"], check=False)
    assert res.returncode == 1 and "error opening" in res.stdout


@pytest.mark.skipif(SKIN is None or not SKIN.exists(), reason="reference fixture not present")
def test_reads_the_reference_fixture(tmp_path):
    out = tmp_path / "in.bin"
    run_cli([1000, 1000, 4, 8, 8, 5, SKIN, SKIN], {"KNNJOIN_DUMP_INPUT": str(out)})
    q, _ = dumped_inputs(out, 1000, 1000, 4)
    want = np.loadtxt(SKIN, max_rows=1000, dtype=np.float32)
    assert np.array_equal(q, want)


@pytest.mark.gpu
def test_cli_join_matches_oracle(tmp_path, oracle, cuda_device):
    x = data.skin_like(6000, seed=9)
    f = tmp_path / "pts.txt"
    np.savetxt(f, x, fmt="%d", delimiter=" ")
    dump = tmp_path / "res.bin"
    res = run_cli([6000, 6000, 3, 60, 60, 50, f, f], {"KNNJOIN_DUMP": str(dump)})
    lines = res.stdout.splitlines()
    assert any(line.startswith("total time ") for line in lines)
    assert any(line.startswith("Total ") for line in lines)
    rec = np.fromfile(dump, dtype=np.dtype([("index", np.int32), ("dist", np.float32)]))
    rec = rec.reshape(6000, 50)
    oi, od = oracle.bruteforce_f64(x, x, 50)
    assert np.array_equal(rec["index"], oi)
    assert np.array_equal(rec["dist"], od.astype(np.float32))
    ik = [line for line in lines if line.startswith("i,k 100 ")]
    assert len(ik) == 50
    parts = ik[3].split()
    assert int(parts[3]) == oi[100, 3] and abs(float(parts[4]) - od[100, 3]) < 1e-5
