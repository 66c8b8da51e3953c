"""Run one join of a named benchmark configuration and print its statistics.

    python -m knn_sweet_b200.workloads c1|c2|c3|c3-small|c4|c4-small|c5 [--form fp32|bf16_refine]
                                       [--repeat N]

  c1        skin-like self-join, N = M = 245,057, d = 3, k = 200, reps 800/800
  c2        N = 1,000,000, M = 100,000, d = 32, k = 32, reps 1000/1000, 3 refinement steps
  c3        N = 2,000,000, M = 200,000, d = 128, k = 100, reps 8192/8192, 4 steps, 1 draw
  c3-small  N = 400,000, M = 40,000, d = 128, k = 100, reps 1600/1600, 4 steps (sized
            for profiler captures: inputs above L2, a few hundred MB on the device)
  c4        4,096 ellipsoid clouds (256..16,384 points), d = 3, per-cloud self-join, k = 16
  c4-small  512 clouds of the same sizes, no autotuning (sized for profiler captures)
  c5        64 blob cloud pairs (2,048..32,768 points), d = 3, k = 8 in both directions,
            forward + backward of the summed loss

Data are the seeded synthetic sets of ``knn_sweet_b200.data``; the inputs are copied
to the GPU before the joins run.  Used to reproduce the figures and profiles of the
benchmark configurations.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import data


def _pair_join(name, q, r, k, form, repeat, **kw):
    import torch
    from .join import knnjoin
    qt = torch.from_numpy(q).cuda()
    rt = qt if r is None else torch.from_numpy(r).cuda()
    for _ in range(repeat):
        _, _, st = knnjoin(qt, None if r is None else rt, k, precision=form, stats=True, **kw)
    print(f"{name} form={form} m={qt.shape[0]} k={k}: total {st.ms_total:.2f} ms "
          f"(build {st.ms_build:.2f}, search {st.ms_search:.2f}), "
          f"{st.dist_evals / qt.shape[0]:.0f} distance evaluations per query, "
          f"{st.refine_fallbacks} fallbacks", flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("workload", choices=["c1", "c2", "c3", "c3-small", "c4", "c4-small", "c5"])
    ap.add_argument("--form", choices=["fp32", "bf16_refine"], default="fp32")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args(argv)
    import torch
    if a.workload == "c1":
        _pair_join("c1", data.skin_like(), None, 200, a.form, a.repeat, qreps=800, sreps=800)
    elif a.workload == "c2":
        r, q = data.config2()
        _pair_join("c2", q, r, 32, a.form, a.repeat, qreps=1000, sreps=1000, lloyd_iters=3)
    elif a.workload == "c3":
        r, q = data.config3()
        _pair_join("c3", q, r, 100, a.form, a.repeat, qreps=8192, sreps=8192, lloyd_iters=4,
                   rep_trials=1)
    elif a.workload == "c3-small":
        r, q = data.gaussian_mix(400_000, 40_000, 128, 800, seed=3, center_kind="normal3",
                                 sigma=0.5)
        _pair_join("c3-small", q, r, 100, a.form, a.repeat, qreps=1600, sreps=1600,
                   lloyd_iters=4)
    elif a.workload in ("c4", "c4-small"):
        from .batched import knnjoin_batched
        small = a.workload == "c4-small"
        pts, off = data.ellipsoid_clouds(nclouds=512 if small else 4096)
        x = torch.from_numpy(pts).cuda()
        for _ in range(a.repeat):
            _, _, st = knnjoin_batched(x, off, k=16, rep_trials=1, autotune=not small,
                                       stats=True)
        print(f"{a.workload} clouds={len(off) - 1} points={x.shape[0]}: total "
              f"{st.ms_total:.2f} ms (build {st.ms_build:.2f}, search {st.ms_search:.2f})",
              flush=True)
    else:
        from .autograd import knn_chamfer_batched
        pairs = data.blob_cloud_pairs()
        xo = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])]).astype(np.int64)
        yo = np.concatenate([[0], np.cumsum([len(p[1]) for p in pairs])]).astype(np.int64)
        x = torch.from_numpy(np.concatenate([p[0] for p in pairs])).cuda().requires_grad_(True)
        y = torch.from_numpy(np.concatenate([p[1] for p in pairs])).cuda().requires_grad_(True)
        for _ in range(a.repeat):
            x.grad = y.grad = None
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            loss = knn_chamfer_batched(x, xo, y, yo, 8)
            loss.backward()
            torch.cuda.synchronize()
            ms = (time.perf_counter() - t0) * 1e3
        print(f"c5 pairs={len(pairs)} points={x.shape[0] + y.shape[0]}: forward+backward "
              f"{ms:.2f} ms, loss {float(loss.detach()):.6g}", flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
