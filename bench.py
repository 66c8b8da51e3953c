#!/usr/bin/env python
"""Benchmark of the exact kNN join (one JSON line on rank 0).

Workload (one step): the exact self-join of a seeded skin-like point set --
N = M = 245,057 integer RGB points (d=3), k = 200, 800 query and 800 reference
representatives -- the reference's sample run shape (run_sample.sh:1) at the
size of its Skin Segmentation table.  Inputs are resident in HBM when a step
starts; a step is the whole join: representative draw, assignment, cluster
sort, bounds, filter and the per-query pruned scan.  L2 is flushed (256 MB
write) before every timed step, outside the timed events.

    python bench.py [--gpus N --steps K --warmup W]        # this build
    python bench.py --impl reference ...                    # CPU reference arm

Multi-GPU (torchrun, one process per GPU): ONE join split across the ranks
("strong" scaling).  Every rank builds the same index from the same points
(the build is deterministic), takes its share of the query clusters --
balanced by estimated work, knn_join_partition_device -- and the result rows
are all-gathered to rank 0 (NCCL) inside the step; the step time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "exact kNN-join queries/s @k=200: BF16+refine vs plain FP32, same neighbor sets"
K = 200
REPS = 800
D = 3
FALLBACK_HBM_GBS = 6650.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=245_057, help="points (default: full size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the precision, d=32, batching and differentiation forms")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip the run of the reference's own CUDA program")
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(pg, value: float, device) -> float:
    """Max of a per-rank float over all ranks (NCCL between GPUs, gloo on CPU);
    every rank calls it at the same point."""
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(world: int, points_per_rank: int, ms_per_step: float) -> float:
    """Whole-job queries/s when every rank joins its own set of points_per_rank
    queries; the step time is the slowest rank's."""
    return world * points_per_rank / (ms_per_step * 1e-3)


def strong_scaling_value(queries: int, ms_per_step: float) -> float:
    """Whole-job queries/s of one join of `queries` queries split across the
    ranks; the step time is the slowest rank's."""
    return queries / (ms_per_step * 1e-3)


def gather_rows(pg, rows, ri, rd, m: int, k: int, device):
    """Rank 0 receives the full (m, k) result of a partitioned join: every rank
    contributes its query rows and their (k) indices and distances, padded to
    the largest part and all-gathered (NCCL between GPUs, gloo on CPU).
    Returns (idx, dist) on rank 0, None on the other ranks; every rank takes
    the same collective steps."""
    import torch
    cnt = torch.tensor([rows.numel()], dtype=torch.int64, device=device)
    pg.all_reduce(cnt, op=pg.ReduceOp.MAX)
    mx = int(cnt.item())
    n = rows.numel()
    pr = torch.full((mx,), -1, dtype=torch.int32, device=device)
    pi = torch.full((mx, k), -1, dtype=torch.int32, device=device)
    pd = torch.zeros((mx, k), dtype=torch.float32, device=device)
    pr[:n] = rows
    pi[:n] = ri
    pd[:n] = rd
    world = pg.get_world_size()
    lr = [torch.empty_like(pr) for _ in range(world)]
    li = [torch.empty_like(pi) for _ in range(world)]
    ld = [torch.empty_like(pd) for _ in range(world)]
    pg.all_gather(lr, pr)
    pg.all_gather(li, pi)
    pg.all_gather(ld, pd)
    if pg.get_rank() != 0:
        return None
    out_i = torch.empty((m, k), dtype=torch.int32, device=device)
    out_d = torch.empty((m, k), dtype=torch.float32, device=device)
    for g in range(world):
        ok = lr[g] >= 0
        sel = lr[g][ok].long()
        out_i[sel] = li[g][ok]
        out_d[sel] = ld[g][ok]
    return out_i, out_d


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            j = json.loads(p.read_text())
            return float(j["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


# ----------------------------------------------------------------------------
# clocks sampled through NVML during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
        0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
        0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
        0x100: "display_clock_setting",
    }

    def __init__(self, device_index: int):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self.ok = False
        self._stop = threading.Event()
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            props = torch.cuda.get_device_properties(device_index)
            h = None
            try:
                bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id,
                                             props.pci_device_id)
                h = nv.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(device_index)
            self.nv, self.h = nv, h
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False

    def _loop(self):
        nv, h = self.nv, self.h
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                try:
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                except AttributeError:
                    r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.reasons |= int(r)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self.ok:
            self._t = threading.Thread(target=self._loop, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        if self.ok:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        names = [n for bit, n in self.REASONS.items() if self.reasons & bit and n != "gpu_idle"]
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


# ----------------------------------------------------------------------------
# CPU baseline: the reference's pruned method restated on the host (oracle)
# ----------------------------------------------------------------------------
def cpu_port_time(x: np.ndarray, sample: int, threads: int, seed: int = 7):
    """Seconds for the full-size join estimated from a bounded sample: the
    port's own timers give the index build on the full set and the scan of
    `sample` random queries; the scan is scaled to all queries."""
    from oracle import oracle as orc
    m = x.shape[0]
    sample = min(sample, m)
    rows = np.random.default_rng(seed).choice(m, sample, replace=False).astype(np.int64)
    _, _, st = orc.port_join(x, x, K, REPS, REPS, qrows=rows, threads=threads)
    t_build, t_scan = st["build_seconds"], max(st["scan_seconds"], 1e-9)
    est = t_build + t_scan * m / sample
    return est, t_build, t_scan


def cpu_sample_size(x: np.ndarray, threads: int, scan_budget_s: float) -> int:
    """Queries whose scan takes about scan_budget_s on the host (pilot run)."""
    m = x.shape[0]
    pilot = min(m, 2000)
    _, _, ts = cpu_port_time(x, pilot, threads, seed=1)
    per_query = ts / pilot
    return int(max(pilot, min(m, scan_budget_s / max(per_query, 1e-9))))


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from knn_sweet_b200 import data
    x = data.skin_like(args.n, seed=1)
    m = x.shape[0]
    cores = host_cores()
    # each step: full index build + a query sample, sized so that the whole
    # run stays within about three minutes
    budget = max(0.2, 150.0 / (args.warmup + args.steps) - 0.7)
    sample = cpu_sample_size(x, cores, budget)
    times = []
    for it in range(args.warmup + args.steps):
        est, tb, ts = cpu_port_time(x, sample, cores, seed=100 + it)
        if it >= args.warmup:
            times.append(est)
    t = statistics.mean(times)
    value = m / t
    desc = (f"index build on all {m} points + pruned scan of {sample} sampled queries per "
            f"step, scaled to {m} queries")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"skin-like self-join N=M={m} d=3 k={K} reps {REPS}/{REPS}",
                   "reference_arm": "CPU restatement of the reference's pruned join "
                                    "(the reference ships no CPU implementation of it)"},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# this build
# ----------------------------------------------------------------------------
def run_ours(args):
    import torch
    import knn_sweet_b200 as ks
    from knn_sweet_b200 import data

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=dev)
        pg = tdist

    x = data.skin_like(args.n, seed=1)
    m = x.shape[0]
    xt = torch.from_numpy(x).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(stats=False):
        if world == 1:
            return ks.knnjoin(xt, None, K, qreps=REPS, sreps=REPS, stats=stats)
        # this rank's part of the one join, then the rows to rank 0
        out = ks.knnjoin_partition(xt, None, K, part=rank, nparts=world, qreps=REPS,
                                   sreps=REPS, stats=stats)
        idx, dist, rows = out[:3]
        rl = rows.long()
        got = gather_rows(pg, rows, idx[rl], dist[rl], m, K, dev)
        res = got if got is not None else (idx, dist)
        return (*res, out[3]) if stats else res

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    # timed region: K steps, per-step CUDA events, L2 flushed before each step
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local)
    with sampler:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            starts[i].record(stream)
            step()
            ends[i].record(stream)
        torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(pg, sum(step_ms), dev)
    ms_per_step = total_ms / args.steps
    value = strong_scaling_value(m, ms_per_step)

    # same steps with the library's own stage events (build / scan split),
    # giving the scan kernel's duration for the roofline
    builds, scans, evals, launches = [], [], [], []
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        _, _, st = step(stats=True)
        builds.append(st.ms_build)
        scans.append(st.ms_search)
        evals.append(st.dist_evals)
        launches.append(st.kernels_launched)
    boundary = {"fp64_rechecks": st.fp64_rechecks, "band_queries": st.band_queries}
    scan_ms = statistics.mean(scans)
    build_ms = statistics.mean(builds)

    # end to end through the public API with host buffers (pinned), copies
    # inside every step (several ranks: the inputs copied in on every rank,
    # the gathered result copied out on rank 0)
    e2e = None
    if not args.no_e2e and world > 1:
        qh = torch.from_numpy(x).pin_memory()
        oi = torch.empty((m, K), dtype=torch.int32).pin_memory()
        od = torch.empty((m, K), dtype=torch.float32).pin_memory()
        wall = []
        for i in range(max(3, args.steps // 3) + 1):
            flush.fill_(i & 0xFF)
            torch.cuda.synchronize(dev)
            pg.barrier()
            t0 = time.perf_counter()
            xd = qh.to(dev, non_blocking=True)
            idx, dist, rows = ks.knnjoin_partition(xd, None, K, part=rank, nparts=world,
                                                   qreps=REPS, sreps=REPS)
            rl = rows.long()
            got = gather_rows(pg, rows, idx[rl], dist[rl], m, K, dev)
            if got is not None:
                oi.copy_(got[0], non_blocking=True)
                od.copy_(got[1], non_blocking=True)
            torch.cuda.synchronize(dev)
            if i > 0:
                wall.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(pg, statistics.mean(wall), dev)
        e2e = {"value": strong_scaling_value(m, e2e_s * 1e3), "unit": "queries/s",
               "h2d_bytes_per_step": int(x.nbytes) * world, "d2h_bytes_per_step": int(m * K * 8),
               "ms_per_step": e2e_s * 1e3}
    if not args.no_e2e and world == 1:
        qh = torch.from_numpy(x).pin_memory().numpy()
        oi = torch.empty((m, K), dtype=torch.int32).pin_memory().numpy()
        od = torch.empty((m, K), dtype=torch.float32).pin_memory().numpy()
        ks.knnjoin(qh, None, K, qreps=REPS, sreps=REPS, out=(oi, od))
        wall = []
        for i in range(max(3, args.steps // 3)):
            flush.fill_(i & 0xFF)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            ks.knnjoin(qh, None, K, qreps=REPS, sreps=REPS, out=(oi, od))
            wall.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(pg, statistics.mean(wall), dev)
        e2e = {"value": strong_scaling_value(m, e2e_s * 1e3), "unit": "queries/s",
               "h2d_bytes_per_step": int(x.nbytes), "d2h_bytes_per_step": int(m * K * 8),
               "ms_per_step": e2e_s * 1e3}

    # the headline join against the FP64 oracle on a sample of queries (every
    # rank joins its part; rank 0 holds the gathered result)
    hi, hd = step()[:2]
    torch.cuda.synchronize(dev)
    if world > 1:
        # the parts' statistics: evaluations summed, stage times the slowest
        tot = torch.tensor([statistics.mean(evals)], dtype=torch.float64, device=dev)
        pg.all_reduce(tot, op=pg.ReduceOp.SUM)
        evals = [float(tot.item())]
        scan_ms = max_over_ranks(pg, scan_ms, dev)
        build_ms = max_over_ranks(pg, build_ms, dev)

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return 0

    peak, peak_kind = measured_peaks()
    bytes_per_query = 4 * D * 2 + 8 * K  # 4d(1 + N/M) + 8k, self-join N = M
    achieved = bytes_per_query * m / (scan_ms * 1e-3) / 1e9
    traffic, warp_inst = None, None
    tp = ROOT / "profiles" / "scan_skin_selfjoin_traffic.json"
    if tp.exists():
        try:
            prof = json.loads(tp.read_text())
            traffic = prof.get("dram_bytes_per_launch")
            warp_inst = prof.get("warp_inst_per_launch")
        except Exception:
            traffic = None
    fp32_flops = statistics.mean(evals) * 3 * D
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic: seeded 2-Gaussian integer RGB mixture standing in for the "
                "Skin Segmentation table",
        "config": {"workload": f"skin-like self-join N=M={m} d=3 k={K} reps {REPS}/{REPS}",
                   "form": "plain FP32 pruned join", "parallelism": (f"query-cluster partition x{world}, results all-gathered to rank 0"
                                   if world > 1 else "one GPU"),
                   "l2": "flushed (256 MB write) before every timed step",
                   "build_ms": build_ms, "scan_ms": scan_ms,
                   "dist_evals_per_query": statistics.mean(evals) / m,
                   "pairs_pruned_frac": 1.0 - statistics.mean(evals) / (m * m),
                   "k_th_boundary": boundary},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "scan_kernel", "peak_source": peak_kind,
                     "bytes_per_query": bytes_per_query,
                     "fp32_tflops": fp32_flops / (scan_ms * 1e-3) / 1e12},
        "gpu_launches": int(statistics.mean(launches)) * args.steps,
        "clocks": sampler.summary(),
    }
    # the bound the scan kernel has: instruction issue.  Warp instructions per
    # launch (one ncu capture of the same launch) over its event-timed
    # duration, against SMs x 4 schedulers x one instruction per clock at the
    # median SM clock of the timed region
    clk = line["clocks"].get("sm_mhz") or line["clocks"].get("sm_max_mhz")
    if warp_inst and clk:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        ach = warp_inst / (scan_ms * 1e-3) / 1e12
        pk = sms * 4 * clk * 1e6 / 1e12
        line["roofline"]["issue"] = {
            "achieved": ach, "peak": pk, "unit": "T warp-instructions/s", "frac": ach / pk,
            "warp_inst_per_launch": warp_inst,
            "warp_inst_per_eval": warp_inst / statistics.mean(evals),
            "peak_source": f"{sms} SMs x 4 issue slots x {clk:.0f} MHz (median under load)"}
    if e2e:
        line["e2e"] = e2e
    line["oracle_err"] = oracle_err(hi.cpu().numpy(), hd.cpu().numpy(), x, x, K,
                                    _sample_rows(m, 2000, 5))
    del hi, hd
    if world == 1 and not args.no_forms:
        line["forms"] = run_forms(torch, dev, flush)
    if world == 1 and not args.no_reference_cuda:
        line["reference_cuda"] = reference_cuda(x)
    if world == 1 and not args.no_cpu_baseline:
        cores = host_cores()
        sample = cpu_sample_size(x, cores, 10.0)
        est, tb, ts = cpu_port_time(x, sample, cores)
        line["cpu_baseline"] = {
            "value": m / est, "unit": "queries/s", "cores": cores, "kind": "port",
            "sample": f"index build on all {m} points ({tb:.2f} s) + pruned scan of "
                      f"{sample} sampled queries ({ts:.2f} s), scaled to {m} queries"}
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


def _time_steps(torch, dev, fn, steps, flush):
    """Mean device time (ms) of `steps` calls of fn, L2 flushed before each."""
    fn()
    torch.cuda.synchronize(dev)
    ms = []
    for i in range(steps):
        flush.fill_(i & 0xFF)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        fn()
        s1.record()
        torch.cuda.synchronize(dev)
        ms.append(s0.elapsed_time(s1))
    return statistics.mean(ms)


# ----------------------------------------------------------------------------
# checks against the FP64 brute-force oracle (after the timed regions; the
# oracle is the checker, never timed)
# ----------------------------------------------------------------------------
def oracle_err(idx, dist, q, r, k, rows, squared=False):
    """Error of a join's rows against the FP64 oracle: the fraction of sampled
    queries whose neighbour set differs, and the largest relative distance
    error (position by position)."""
    from oracle import oracle as orc
    oi, od = orc.bruteforce_f64(q, r, k, qrows=np.asarray(rows, np.int64), threads=host_cores())
    return compare_to_oracle(np.asarray(idx)[rows], np.asarray(dist)[rows], oi, od, squared)


def compare_to_oracle(idx, dist, oi, od, squared=False):
    idx = np.asarray(idx)
    dist = np.asarray(dist, np.float64)
    if squared:
        dist = np.sqrt(dist)
    sets = (np.sort(idx, 1) != np.sort(oi, 1)).any(1)
    fin = np.isfinite(od)
    both = np.array_equal(np.isfinite(dist), fin)
    rel = np.abs(dist[fin] - od[fin]) / np.maximum(od[fin], 1e-30)
    return {"queries": int(idx.shape[0]), "set_mismatch_frac": float(sets.mean()),
            "max_rel_dist_err": float(rel.max()) if rel.size else 0.0,
            "missing_slots_agree": bool(both)}


def _merge_errs(errs, what):
    n = sum(e["queries"] for e in errs)
    return {"sample": what, "queries": n,
            "set_mismatch_frac": sum(e["set_mismatch_frac"] * e["queries"] for e in errs)
            / max(1, n),
            "max_rel_dist_err": max(e["max_rel_dist_err"] for e in errs),
            "missing_slots_agree": all(e["missing_slots_agree"] for e in errs)}


def _sample_rows(m, count, seed):
    return np.sort(np.random.default_rng(seed).choice(m, min(count, m), replace=False))


def _pair_forms(torch, dev, flush, r, q, k, kw, steps, sample, seed):
    """Plain FP32 and BF16+refine on the same inputs and representatives: time,
    statistics, agreement of the two forms and each form's oracle error."""
    import knn_sweet_b200 as ks
    rt, qt = torch.from_numpy(r).to(dev), torch.from_numpy(q).to(dev)
    m = qt.shape[0]
    res, forms = {}, {}
    for prec in ("fp32", "bf16_refine"):
        o = (torch.empty((m, k), dtype=torch.int32, device=dev),
             torch.empty((m, k), dtype=torch.float32, device=dev))
        ms = _time_steps(torch, dev, lambda: ks.knnjoin(qt, rt, k, precision=prec, out=o, **kw),
                         steps, flush)
        _, _, st = ks.knnjoin(qt, rt, k, precision=prec, out=o, stats=True, **kw)
        res[prec] = o
        forms[prec] = {"queries_per_s": m / (ms * 1e-3), "ms_per_step": ms,
                       "build_ms": st.ms_build, "search_ms": st.ms_search,
                       "dist_evals_per_query": st.dist_evals / m,
                       "fp64_rechecks": st.fp64_rechecks, "band_queries": st.band_queries,
                       "fallback_queries": st.refine_fallbacks}
    a, b = res["fp32"][0], res["bf16_refine"][0]
    same = (torch.sort(a, 1)[0] == torch.sort(b, 1)[0]).all(1).float().mean().item()
    torch.cuda.synchronize(dev)
    del rt, qt
    rows = _sample_rows(m, sample, seed)
    from oracle import oracle as orc
    oi, od = orc.bruteforce_f64(q, r, k, qrows=rows.astype(np.int64), threads=host_cores())
    for prec in forms:
        forms[prec]["oracle_err"] = compare_to_oracle(res[prec][0][rows].cpu().numpy(),
                                                      res[prec][1][rows].cpu().numpy(), oi, od)
    return forms, same


def form_precision(torch, dev, flush, steps):
    """Precision form (2,000,000 reference / 200,000 query points, d=128,
    k=100, seeded mixture of 4,096 Gaussians): plain FP32 vs BF16+refine on the
    same representatives."""
    from knn_sweet_b200 import data
    r, q = data.config3()
    k = 100
    # the representatives are refined (4 centroid steps with the cluster
    # split), so one random draw seeds them as well as the best of ten
    forms, same = _pair_forms(torch, dev, flush, r, q, k,
                              dict(qreps=8192, sreps=8192, lloyd_iters=4, rep_trials=1), steps,
                              500, 33)
    return {"workload": f"N={r.shape[0]} M={q.shape[0]} d=128 k={k} reps 8192/8192 lloyd 4, "
                        "1 draw trial, synthetic 4,096-Gaussian mixture",
            "fp32": forms["fp32"], "bf16_refine": forms["bf16_refine"],
            "same_neighbor_sets": same,
            "bf16_over_fp32": forms["bf16_refine"]["queries_per_s"] / forms["fp32"]["queries_per_s"]}


def form_c2(torch, dev, flush, steps):
    """Higher-dimension plain join (1,000,000 reference / 100,000 query points,
    d=32, k=32, 1,000 representatives per side, seeded mixture of 1,000
    Gaussians), both forms."""
    from knn_sweet_b200 import data
    r, q = data.config2()
    k = 32
    forms, same = _pair_forms(torch, dev, flush, r, q, k,
                              dict(qreps=1000, sreps=1000, lloyd_iters=3), steps, 1000, 22)
    return {"workload": f"N={r.shape[0]} M={q.shape[0]} d=32 k={k} reps 1000/1000 lloyd 3, "
                        "10 draw trials, synthetic 1,000-Gaussian mixture",
            "fp32": forms["fp32"], "bf16_refine": forms["bf16_refine"],
            "same_neighbor_sets": same,
            "bf16_over_fp32": forms["bf16_refine"]["queries_per_s"] / forms["fp32"]["queries_per_s"]}


def form_batching(torch, dev, flush, steps):
    """Batching form (4,096 ellipsoid clouds of 256..16,384 points, d=3,
    per-cloud self-join k=16): one graph-replayed batched call vs one plain call
    per cloud; oracle error over 16 sampled whole clouds."""
    import knn_sweet_b200 as ks
    from knn_sweet_b200 import data
    from knn_sweet_b200.batched import BatchedJoinGraph
    pts, off = data.ellipsoid_clouds()
    x = torch.from_numpy(pts).to(dev)
    mq, kb = x.shape[0], 16
    # one representative draw per cloud (best of 10 draws: 75.9 against 74.5
    # ms, same evaluations and sets), for the per-cloud calls as well
    g = BatchedJoinGraph(off, d=3, k=kb, rep_trials=1)
    g(x)
    torch.cuda.synchronize(dev)
    ms_b = _time_steps(torch, dev, lambda: g(x), steps, flush)
    bi, bd = g.idx.clone(), g.dist.clone()
    oi = torch.empty((mq, kb), dtype=torch.int32, device=dev)
    od = torch.empty((mq, kb), dtype=torch.float32, device=dev)
    bounds = [(int(off[c]), int(off[c + 1])) for c in range(len(off) - 1)]

    def per_cloud():
        for a0, a1 in bounds:
            ks.knnjoin(x[a0:a1], None, kb, rep_trials=1, out=(oi[a0:a1], od[a0:a1]))
    ms_p = _time_steps(torch, dev, per_cloud, 1, flush)
    same_b = (torch.sort(oi, 1)[0] == torch.sort(bi, 1)[0]).all(1).float().mean().item()
    bi, bd = bi.cpu().numpy(), bd.cpu().numpy()
    from oracle import oracle as orc
    errs = []
    for c in _sample_rows(len(bounds), 16, 44):
        a0, a1 = bounds[c]
        ci, cd = orc.bruteforce_f64(pts[a0:a1], pts[a0:a1], kb, threads=host_cores())
        errs.append(compare_to_oracle(bi[a0:a1], bd[a0:a1], ci, cd))
    return {"workload": f"{len(bounds)} ellipsoid clouds, {mq} points, d=3, per-cloud "
                        f"self-join k={kb}",
            "batched_graph": {"queries_per_s": mq / (ms_b * 1e-3), "ms_per_step": ms_b,
                              "oracle_err": _merge_errs(errs, "16 whole clouds")},
            "per_cloud_calls": {"queries_per_s": mq / (ms_p * 1e-3), "ms_per_step": ms_p},
            "same_neighbor_sets": same_b, "batched_over_per_cloud": ms_p / ms_b}


def form_differentiation(torch, dev, flush, steps):
    """Differentiation form (64 blob cloud pairs of 2,048..32,768 points, d=3):
    forward + hand-written backward of the summed k nearest squared distances in
    both directions (k=8, and the k=1 Chamfer loss).  Checked on 16 sampled
    pairs: forward neighbour sets against the FP64 oracle, and the gradient
    against the FP64 gradient of the same loss over the oracle's pairs."""
    from knn_sweet_b200 import data
    from knn_sweet_b200.autograd import knn_chamfer_batched, knn_dist2_batched
    pairs = data.blob_cloud_pairs()
    xo = np.concatenate([[0], np.cumsum([len(p[0]) for p in pairs])]).astype(np.int64)
    yo = np.concatenate([[0], np.cumsum([len(p[1]) for p in pairs])]).astype(np.int64)
    xs = np.concatenate([p[0] for p in pairs])
    ys = np.concatenate([p[1] for p in pairs])
    x = torch.from_numpy(xs).to(dev).requires_grad_(True)
    y = torch.from_numpy(ys).to(dev).requires_grad_(True)
    npts = x.shape[0] + y.shape[0]
    out = {"workload": f"{len(pairs)} blob cloud pairs, {npts} points, d=3, loss = sum of "
                       "k nearest squared distances in both directions, forward + backward"}
    for k in (8, 1):
        def fwd_bwd():
            x.grad = y.grad = None
            knn_chamfer_batched(x, xo, y, yo, k).backward()
        ms = _time_steps(torch, dev, fwd_bwd, steps, flush)
        out[f"k{k}"] = {"queries_per_s": npts / (ms * 1e-3), "ms_per_step": ms}
    # checks (k = 8)
    k = 8
    x.grad = y.grad = None
    knn_chamfer_batched(x, xo, y, yo, k).backward()
    gx, gy = x.grad.double().cpu().numpy(), y.grad.double().cpu().numpy()
    with torch.no_grad():
        dxy, ixy = knn_dist2_batched(x.detach(), xo, y.detach(), yo, k)
        dyx, iyx = knn_dist2_batched(y.detach(), yo, x.detach(), xo, k)
    ixy, iyx = ixy.cpu().numpy(), iyx.cpu().numpy()
    dxy, dyx = dxy.cpu().numpy(), dyx.cpu().numpy()
    from oracle import oracle as orc
    errs, gerr = [], 0.0
    for c in _sample_rows(len(pairs), 16, 55):
        xa, xb, ya, yb = xo[c], xo[c + 1], yo[c], yo[c + 1]
        px, py = xs[xa:xb].astype(np.float64), ys[ya:yb].astype(np.float64)
        oxy, dxy_o = orc.bruteforce_f64(xs[xa:xb], ys[ya:yb], k, threads=host_cores())
        oyx, dyx_o = orc.bruteforce_f64(ys[ya:yb], xs[xa:xb], k, threads=host_cores())
        errs.append(compare_to_oracle(ixy[xa:xb], dxy[xa:xb], oxy, dxy_o, squared=True))
        errs.append(compare_to_oracle(iyx[ya:yb], dyx[ya:yb], oyx, dyx_o, squared=True))
        # FP64 gradient of the pair's loss over the oracle's neighbour pairs
        rgx, rgy = np.zeros_like(px), np.zeros_like(py)
        dv = px[:, None, :] - py[oxy]                  # x_i - y_j
        rgx += 2 * dv.sum(1)
        np.add.at(rgy, oxy.ravel(), -2 * dv.reshape(-1, 3))
        dv = py[:, None, :] - px[oyx]                  # y_j - x_i
        rgy += 2 * dv.sum(1)
        np.add.at(rgx, oyx.ravel(), -2 * dv.reshape(-1, 3))
        scale = max(np.abs(rgx).max(), np.abs(rgy).max(), 1e-30)
        gerr = max(gerr, np.abs(gx[xa:xb] - rgx).max() / scale,
                   np.abs(gy[ya:yb] - rgy).max() / scale)
    out["k8"]["oracle_err"] = _merge_errs(errs, "16 pairs, both directions")
    out["k8"]["grad_max_err_rel_to_max"] = float(gerr)
    return out


def run_forms(torch, dev, flush, steps=3):
    """The precision, batching and differentiation forms beside the plain FP32
    join, and the d = 32 plain join; each with its error against the FP64
    oracle."""
    out = {"precision": form_precision(torch, dev, flush, steps)}
    torch.cuda.empty_cache()
    out["c2"] = form_c2(torch, dev, flush, steps)
    torch.cuda.empty_cache()
    out["batching"] = form_batching(torch, dev, flush, steps)
    torch.cuda.empty_cache()
    out["differentiation"] = form_differentiation(torch, dev, flush, steps)
    torch.cuda.empty_cache()
    return out


def reference_cuda(x: np.ndarray):
    """The reference's own CUDA program (oracle/_ref/knnjoin_ref, built from the
    reference's sources by oracle/build_ref.sh) on the same points written as its
    text input, reps 800/800, K=200: its own "total time" line
    (src/knnjoin.cu:1136, which covers knnjoin.cu:274-1135 and so excludes its
    H2D copies and representative draw) and the wall time of its process."""
    ref = ROOT / "oracle" / "_ref" / "knnjoin_ref"
    if not ref.exists():
        return {"unavailable": "oracle/_ref/knnjoin_ref not built (oracle/build_ref.sh)"}
    import tempfile
    from oracle.compare_ref import agreement, run_reference
    try:
        with tempfile.TemporaryDirectory() as td:
            ri, rd, info = run_reference(x, K, REPS, Path(td), timeout=300)
    except Exception as e:  # reported, not raised: the arm is informational
        return {"unavailable": f"reference run failed: {str(e)[:200]}"}
    rows = _sample_rows(x.shape[0], 1000, 12)
    from oracle import oracle as orc
    oi, od = orc.bruteforce_f64(x, x, K, qrows=rows.astype(np.int64), threads=host_cores())
    return {"total_time_ms": info["total_time_s"] * 1e3 if info["total_time_s"] else None,
            "process_wall_s": info["wall_s"], "dist_evals": info["dist_evals"],
            "coverage": "its own total time: clustering, bounds, filter and scan of the GPU "
                        "program (knnjoin.cu:274-1135); excludes its text parsing, H2D copies "
                        "and representative draw, which this build's step includes",
            "vs_fp64_oracle": agreement(ri[rows], rd[rows], oi, od)}


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
