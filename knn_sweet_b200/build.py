"""In-tree build of libknnsweet.so (sm_100a) and the `knnjoin` command line.

    python -m knn_sweet_b200.build          # incremental
    python -m knn_sweet_b200.build --force  # rebuild everything

Objects go to knn_sweet_b200/_build/, the library to knn_sweet_b200/lib/ and
the command line to knn_sweet_b200/bin/.  nvcc cross-compiles for sm_100a on a
machine without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
BINDIR = PKG / "bin"
LIB = LIBDIR / "libknnsweet.so"
CLI = BINDIR / "knnjoin"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-Wall", "-I", str(ROOT / "include"),
]

CU_SOURCES = ["api.cu", "build_index.cu", "scan.cu", "backward.cu", "noalloc.cu", "assign_tc.cu", "batched.cu",
              "tile_search.cu", "sharded.cu"]
HEADERS = ["common.cuh", "kernels.cuh", "glibc_rand.h", "tc_common.cuh", "bounds.cuh",
           "warp_select.cuh", "pipeline.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    BINDIR.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "knnsweet.h"]
    nv = nvcc()
    objs = []
    todo = []
    for src in CU_SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [CSRC / src] + headers):
            todo.append([nv, *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        for cmd, fut in [(c, ex.submit(_run, c)) for c in todo]:
            if verbose:
                print(" ".join(cmd))
            fut.result()
    if force or todo or _stale(LIB, objs):
        _run([nv, *ARCH, "-shared", "-o", str(LIB), *map(str, objs)])
    cli_src = CSRC / "knnjoin_cli.cpp"
    if cli_src.exists() and (force or _stale(CLI, [cli_src, LIB] + headers)):
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-I", str(ROOT / "include"),
              str(cli_src), "-o", str(CLI), f"-L{LIBDIR}", "-lknnsweet",
              "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    lib = build(force=args.force, verbose=args.verbose)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
