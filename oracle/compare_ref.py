"""TEST INFRASTRUCTURE ONLY: runs the reference's own CUDA program
(oracle/_ref/knnjoin_ref, built by oracle/build_ref.sh) on seeded skin-like
points and either

  --golden OUT.npz   saves its full result (the IndexDist array captured by
                     oracle/ref_shim.so) as a small fixture, or
  --compare          compares a run with this build's join and the FP64
                     oracle and prints one JSON line: the reference's own
                     "total time", the wall time of its process, this build's
                     join time on the same points, and agreement figures.

The reference keeps tied neighbours in a nondeterministic order and two of its
bounds can drop true neighbours (defects B1, B2), so agreement is reported as:
  dist_equal   queries whose K sorted distances equal the oracle's
  set_equal    queries whose index sets equal the oracle's after removing the
               points at exactly the K-th distance
  kth_worse    queries whose K-th distance exceeds the oracle's (missed points)
Run on a GPU machine: python oracle/compare_ref.py --compare --n 245057 --k 200
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
# run as a script, sys.path[0] is this folder, where oracle.py would shadow
# the `oracle` package
sys.path[0] = str(ROOT)

REF_BIN = HERE / "_ref" / "knnjoin_ref"
SHIM = HERE / "_ref" / "ref_shim.so"


def run_reference(x: np.ndarray, k: int, reps: int, workdir: Path, timeout: int = 900):
    n, d = x.shape
    txt = workdir / "points.txt"
    np.savetxt(txt, x, fmt="%d" if np.all(x == np.rint(x)) else "%.9g", delimiter=" ")
    dump = workdir / "ref_result.bin"
    env = dict(os.environ)
    env.update({"LD_PRELOAD": str(SHIM), "MALLOC_PERTURB_": "255",
                "KNN_REF_DUMP_BYTES": str(n * k * 8), "KNN_REF_DUMP_PATH": str(dump)})
    cmd = [str(REF_BIN), str(n), str(n), str(d), str(reps), str(reps), str(k), str(txt),
           str(txt)]
    t0 = time.perf_counter()
    res = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
    wall = time.perf_counter() - t0
    if res.returncode != 0:
        raise RuntimeError(f"reference failed ({res.returncode}):\n{res.stdout[-2000:]}\n"
                           f"{res.stderr[-2000:]}")
    m = re.search(r"total time ([0-9.eE+-]+)", res.stdout)
    total = float(m.group(1)) if m else None
    tot = re.search(r"^Total (\d+)", res.stdout, re.M)
    rec = np.fromfile(dump, dtype=np.dtype([("index", np.int32), ("dist", np.float32)]))
    rec = rec.reshape(n, k)
    return rec["index"].copy(), rec["dist"].copy(), {
        "total_time_s": total, "wall_s": wall, "dist_evals": int(tot.group(1)) if tot else None,
        "shim_log": [ln for ln in res.stderr.splitlines() if ln.startswith("[ref_shim]")][:4]}


def agreement(ri, rd, oi, od):
    """Per-query agreement of the reference (ri, rd) with the oracle (oi, od)."""
    od32 = od.astype(np.float32)
    rd_sorted = np.sort(rd, axis=1)
    dist_equal = np.all(rd_sorted == od32, axis=1)
    kth = od32[:, -1:]
    set_equal = np.empty(len(ri), bool)
    for i in range(len(ri)):
        a = set(ri[i][rd[i] < kth[i, 0]].tolist())
        b = set(oi[i][od32[i] < kth[i, 0]].tolist())
        set_equal[i] = a == b
    kth_worse = rd_sorted[:, -1] > od32[:, -1]
    return {"dist_equal": float(dist_equal.mean()), "set_equal": float(set_equal.mean()),
            "kth_worse": float(kth_worse.mean()), "queries": int(len(ri))}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--k", type=int, default=32)
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--golden", type=Path)
    ap.add_argument("--compare", action="store_true")
    ap.add_argument("--sample", type=int, default=2000, help="oracle rows for --compare")
    args = ap.parse_args(argv)

    from knn_sweet_b200 import data
    from oracle import oracle as orc

    x = data.skin_like(args.n, seed=args.seed)
    with tempfile.TemporaryDirectory() as td:
        ri, rd, info = run_reference(x, args.k, args.reps, Path(td))
    if args.golden:
        np.savez_compressed(args.golden, x=x, k=np.array(args.k), reps=np.array(args.reps),
                            seed=np.array(args.seed), ref_idx=ri, ref_dist=rd)
        print(json.dumps({"golden": str(args.golden), **info}))
        return 0
    if args.compare:
        import torch
        import knn_sweet_b200 as ks
        xt = torch.from_numpy(x).cuda()
        for _ in range(3):
            ks.knnjoin(xt, None, args.k, qreps=args.reps, sreps=args.reps)
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            oi_t, od_t = ks.knnjoin(xt, None, args.k, qreps=args.reps, sreps=args.reps)
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) / 1e3)
        ours_i, ours_d = oi_t.cpu().numpy(), od_t.cpu().numpy()
        rows = np.random.default_rng(0).choice(args.n, min(args.sample, args.n), replace=False)
        oi, od = orc.bruteforce_f64(x, x, args.k, qrows=rows)
        ours_exact = bool(np.array_equal(ours_i[rows], oi) and
                          np.array_equal(ours_d[rows], od.astype(np.float32)))
        out = {"n": args.n, "k": args.k, "reps": args.reps, "reference": info,
               "ours_join_s_median": float(np.median(ts)), "ours_exact_on_sample": ours_exact,
               "reference_vs_oracle": agreement(ri[rows], rd[rows], oi, od),
               "speedup_vs_reference_total_time":
                   (info["total_time_s"] / float(np.median(ts))) if info["total_time_s"] else None}
        print(json.dumps(out))
        return 0
    print(json.dumps(info))
    return 0


if __name__ == "__main__":
    sys.exit(main())
