#!/usr/bin/env python3
"""Builds the engine's shared library in-tree: lib/libbk_b200.so (sm_100a only).

    python bernasconi-krylov_b200/build.py [--verbose]

nvcc cross-compiles without a GPU. The library exports the C ABI declared in
include/bk_engine.h and links only the CUDA runtime (the driver's tensor-map
encoder is resolved at run time through cudaGetDriverEntryPoint).
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libbk_b200.so")
SOURCES = ["csrc/bk_engine.cu", "csrc/bk_noalloc.cu"]
HEADERS = ["csrc/bk_device.cuh", "csrc/bk_fused.cuh", "csrc/bk_aux.cuh", "csrc/bk_persist.cuh", "csrc/bk_adjoint.cuh", "csrc/bk_lanczos.cuh", "csrc/bk_s23.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp", "-shared", "-ccbin", "/usr/bin/g++",
         "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(HERE, "csrc")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = SOURCES + HEADERS + [os.path.join(ROOT, "include", "bk_engine.h")]
    return all(os.path.getmtime(os.path.join(HERE, d) if not os.path.isabs(d) else d) <= t for d in deps)


def build(verbose=False, force=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + \
        [os.path.join(HERE, s) for s in SOURCES] + ["-o", LIB, "-lcudart", "-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building " + LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))
