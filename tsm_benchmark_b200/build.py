#!/usr/bin/env python3
"""Builds the CUDA library in-tree: tsm_benchmark_b200/libtsm_b200.so.

    python -m tsm_benchmark_b200.build [--jobs N] [--force] [--ptxas-verbose]

Every ``.cu`` under ``csrc/`` (including the generator's output in
``csrc/generated/``) is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) into ``_build/`` and linked
into one shared library whose exported symbols are the C ABI of
``include/tsm.h``.  Objects are rebuilt when their source or any header is
newer.  nvcc cross-compiles, so no GPU is needed.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libtsm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", f"-I{os.path.join(ROOT, 'include')}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found (CUDA toolkit required to build the library)")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "generated", "*.cu")))


def headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _obj_for(src: str) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "__")
    return os.path.join(BUILD, rel[:-3] + ".o")


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, ptxas_verbose: bool) -> tuple[str, str]:
    obj = _obj_for(src)
    cmd = [nvcc(), *NVCC_FLAGS, "-c", src, "-o", obj]
    if ptxas_verbose:
        cmd[1:1] = ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(jobs: int | None = None, force: bool = False, ptxas_verbose: bool = False, quiet: bool = False) -> str:
    """Compiles and links; returns the library path."""
    from . import codegen  # keep csrc/generated in step with the generator

    files = codegen.render(codegen.default_variants(), codegen.load_tuned())
    if not codegen.is_current(files):
        codegen.write(files)
    os.makedirs(BUILD, exist_ok=True)
    hdrs = headers()
    srcs = sources()
    todo = [s for s in srcs if force or ptxas_verbose or _stale(_obj_for(s), [s, *hdrs])]
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
    logs = []
    if todo:
        if not quiet:
            print(f"[tsm build] compiling {len(todo)} of {len(srcs)} sources with {jobs} jobs", flush=True)
        with cf.ThreadPoolExecutor(jobs) as ex:
            for obj, log in ex.map(lambda s: _compile(s, ptxas_verbose), todo):
                logs.append((obj, log))
    objs = [_obj_for(s) for s in srcs]
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", *ARCH, "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if ptxas_verbose:
        for obj, log in logs:
            print(f"== {os.path.basename(obj)}\n{log}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="build libtsm_b200.so for sm_100a")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true", help="print registers / spills / smem per kernel")
    args = ap.parse_args(argv)
    path = build(args.jobs, args.force, args.ptxas_verbose)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
