"""The multi-rank path of bench.py on CPU: two gloo ranks (one process each, as
torchrun would start them) agree on the max-over-ranks step time and on the
whole-job value, and the reference arm's non-zero ranks exit without work."""
import json
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    local_ms = 10.0 * (rank + 1)          # rank 1 is the slow one
    ms = bench.max_over_ranks(dist, local_ms, "cpu")
    value = bench.weak_scaling_value(world, 1000, ms)
    rc = 0
    if rank != 0:
        rc = bench.main(["--impl", "reference", "--gpus", str(world)])
    dist.barrier()
    dist.destroy_process_group()
    Path(out_dir, f"rank{rank}.json").write_text(
        json.dumps({"rank": bench.dist_env()[0], "ms": ms, "value": value, "rc": rc}))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_timing(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [json.loads(Path(tmp_path, f"rank{r}.json").read_text()) for r in range(world)]
    for r, x in enumerate(res):
        assert x["rank"] == r
        assert x["ms"] == 20.0                      # the slowest rank's time, everywhere
        assert x["value"] == pytest.approx(2 * 1000 / 0.020)
        assert x["rc"] == 0


def _gather_worker(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    m, k = 11, 3
    # uneven parts, as the work-balanced partition gives: rank 0 takes the
    # rows divisible by 3, rank 1 the rest
    rows = torch.tensor([i for i in range(m) if (i % 3 == 0) == (rank == 0)], dtype=torch.int32)
    ri = (rows[:, None] * 10 + torch.arange(k, dtype=torch.int32)[None, :]).to(torch.int32)
    rd = ri.to(torch.float32) / 4
    got = bench.gather_rows(dist, rows, ri, rd, m, k, "cpu")
    ok = True
    if rank == 0:
        want = torch.arange(m, dtype=torch.int32)[:, None] * 10 + torch.arange(k)[None, :]
        ok = bool(torch.equal(got[0], want.to(torch.int32))
                  and torch.equal(got[1], want.to(torch.float32) / 4))
    else:
        ok = got is None
    ms = bench.max_over_ranks(dist, 1.0 + rank, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    Path(out_dir, f"g{rank}.json").write_text(json.dumps(
        {"ok": ok, "value": bench.strong_scaling_value(m, ms)}))


@pytest.mark.timeout(120)
def test_partitioned_join_rows_gathered_to_rank0(tmp_path):
    """The multi-GPU bench step: each rank's part of one join (uneven row
    sets) all-gathered and assembled into the whole result on rank 0; the
    whole-job value is the query count over the slowest rank's time."""
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_gather_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        x = json.loads(Path(tmp_path, f"g{r}.json").read_text())
        assert x["ok"]
        assert x["value"] == pytest.approx(11 / 0.002)
