"""Build libmxcb200.so in-tree for sm_100a (nvcc, no torch extension machinery).

Usage: python -m mxc_b200.build [--jobs N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmxcb200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

SOURCES = ["plan.cpp", "k_gen.cu", "k_basis.cu", "k_gemm.cu", "k_tc.cu", "k_gram.cu", "k_sketch.cu", "k_mf.cu", "k_bf16.cu", "k_lu.cu", "k_vec.cu", "h2dev.cu",
           "h2_solver.cpp"]
# The reference's command-line driver on this library (C++ host code only).
CLI_SRC = os.path.join(CSRC, "lorasp.cpp")
CLI = os.path.join(HERE, "lorasp")


def _compile(src: str, force: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".hpp", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "h2dev.h"))
    deps.append(os.path.join(ROOT, "include", "mxc_b200", "h2_solver.hpp"))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [NVCC] + ARCH + FLAGS + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + FLAGS + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj


def build(jobs: int = 8, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), SOURCES))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    deps = [CLI_SRC, LIB, os.path.join(ROOT, "include", "mxc_b200", "h2_solver.hpp")]
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(d) for d in deps):
        cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), CLI_SRC, "-o", CLI, "-L" + HERE,
               "-lmxcb200", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("lorasp build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    if verbose:
        print("built", LIB, CLI)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(a.jobs, a.force, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
