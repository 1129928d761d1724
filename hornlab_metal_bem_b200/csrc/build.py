"""Build libhbem.so (sm_100a) in-tree from the CUDA sources next to this file.

    python -m hornlab_metal_bem_b200.csrc.build [--jobs N] [--verbose]

Each translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into ``_build/``
(objects are cached by source/header mtime) and linked into
``hornlab_metal_bem_b200/libhbem.so``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
REPO = PKG.parent
OUT = PKG / "libhbem.so"
BUILD = REPO / "_build" / "hbem"
SOURCES = ["session.cu", "assemble.cu", "field.cu", "lu.cu", "gemm.cu", "sweep.cu", "aperture.cu", "adjoint.cu", "fp64.cu", "near.cu"]
HEADERS = ["hbem_internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", str(REPO / "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime() -> float:
    files = [HERE / h for h in HEADERS] + [REPO / "include" / "hbem.h"]
    return max(f.stat().st_mtime for f in files)


def _compile(src: str, verbose: bool, extra: list[str]) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    s = HERE / src
    if obj.exists() and obj.stat().st_mtime >= max(s.stat().st_mtime, _deps_mtime()) and not extra:
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(s), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr.strip():
        print(res.stderr, flush=True)
    return obj


def build(jobs: int | None = None, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(SOURCES))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose or ptxas_verbose, extra), SOURCES))
    newest = max(o.stat().st_mtime for o in objs)
    if not OUT.exists() or OUT.stat().st_mtime < newest or extra:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args(argv)
    out = build(a.jobs, a.verbose, a.ptxas_verbose)
    print(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
