"""Compile ``libdwg_b200.so`` (all CUDA sources, sm_100a) in-tree with nvcc.

Usage: ``python -m dwg_b200.build [--force] [--jobs N]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdwg_b200.so")
CLI_SRC = os.path.join(HERE, "cli", "dwg_cuda.cpp")
CLI = os.path.join(HERE, "bin", "DWG_CUDA")
COUNTER_SRC = os.path.join(CSRC, "launch_counter.cpp")
COUNTER = os.path.join(HERE, "liblaunch_counter.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I" + os.path.join(ROOT, "include"),
]

# per-file additions: the PCA normals and point areas evaluate the oracle's
# FP64 sequence operation by operation, so nothing is fused into an FMA
FILE_FLAGS = {"areas.cu": ["-fmad=false"]}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    hdrs = headers()
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            todo.append((s, o))
    nv = nvcc()

    def compile_one(so):
        s, o = so
        cmd = [nv] + NVCC_FLAGS + FILE_FLAGS.get(os.path.basename(s), []) + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(s)}:\n{r.stdout}\n{r.stderr}")
        return r.stderr

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for msg in ex.map(compile_one, todo):
                if verbose and msg:
                    print(msg, file=sys.stderr)
    if force or todo or _stale(LIB, objs):
        # static CUDA runtime: the library does not depend on whichever
        # libcudart the host process (e.g. torch) has loaded
        cmd = [nv] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_cli(force)
    build_counter(force)
    return LIB


def build_counter(force: bool = False) -> str:
    """Kernel launch census used by bench.py (CUPTI activity records)."""
    if force or _stale(COUNTER, [COUNTER_SRC]):
        cupti_lib = os.path.join(CUDA_HOME, "targets", "x86_64-linux", "lib")
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + os.path.join(CUDA_HOME, "include"),
               COUNTER_SRC, "-o", COUNTER, "-L" + cupti_lib, "-lcupti", "-Wl,-rpath," + cupti_lib]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"launch counter build failed:\n{r.stdout}\n{r.stderr}")
    return COUNTER


def build_cli(force: bool = False) -> str:
    """DWG_CUDA command line tool, linked against libdwg_b200.so (rpath $ORIGIN/..)."""
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    deps = [CLI_SRC, LIB] + headers()
    if force or _stale(CLI, deps):
        cmd = [nvcc(), "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), CLI_SRC, "-o", CLI,
               "-L" + HERE, "-ldwg_b200", "-Xlinker", "-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"DWG_CUDA build failed:\n{r.stdout}\n{r.stderr}")
    return CLI


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.verbose))


if __name__ == "__main__":
    main()
