"""Builds the sm_100a library in-tree: pcr_b200/lib/libpcr_b200.so (the C ABI
of include/pcr_cuda.h) and the `pcr-render` CLI next to it.

    python -m pcr_b200.build [--force]

nvcc cross-compiles for sm_100a without a GPU.  Host code is built with
-ffp-contract=off so the scene constants it computes (plane dot products,
triangle edges, fit coefficients, BVH boxes) are bit-equal to the
reference's; device intersection code uses explicit round-to-nearest
intrinsics for the same reason.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpcr_b200.so")
CLI = os.path.join(LIBDIR, "pcr-render")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["engine.cu", "bvh_build.cu", "scene.cpp", "capi.cpp"]
HEADERS = ["layout.h", "device.cuh", "kernels.cuh", "engine.h", "scene.h", "bvh_build.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [
        os.path.join(HERE, "..", "include", "pcr_cuda.h"), __file__]
    if force or not _newer(LIB, deps):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-ccbin", "/usr/bin/g++", "-o", LIB] + [os.path.join(CSRC, f) for f in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src) and (force or not _newer(CLI, [cli_src, LIB])):
        cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-ffp-contract=off", "-o", CLI, cli_src,
               os.path.join(CSRC, "cuda_renderer.cpp"), "-I", os.path.join(HERE, "..", "include"),
               "-I", "/usr/local/cuda/include", "-L", LIBDIR, "-lpcr_b200", "-Wl,-rpath,$ORIGIN", "-lz",
               "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
