"""Builds libumap_b200.so in-tree: CUDA kernels for sm_100a (nvcc) + C++ host (g++).

Usage: python umap-rs_b200/build.py [--force] [--verbose]

The library links the CUDA runtime statically, so it loads on a machine without a GPU
(compute calls then return UMAP_ERR_CUDA) and carries no torch dependency.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "umap_b200", "libumap_b200.so")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
             "-I" + INCLUDE, "-I" + CSRC, "-I" + os.path.join(CUDA_HOME, "include")]


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(h) for h in hs) if hs else 0


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    return os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_mtime)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")
    if verbose and (p.stdout or p.stderr):
        sys.stdout.write(p.stdout + p.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = sources()
    hm = _headers_mtime()
    jobs, objs = [], []
    for f in cu:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(src, obj, hm):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            jobs.append([NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", obj])
    for f in cpp:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(src, obj, hm):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda c: _run(c, verbose or ptxas_verbose), jobs))
    if jobs or force or not os.path.exists(OUT):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs +
             ["-lrt", "-lpthread", "-ldl"], verbose)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/smem usage")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas))
