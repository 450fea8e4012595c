"""Builds the native libraries of fir_b200 in-tree.

* ``fir_b200/lib/libfir_cuda.so`` -- the C ABI of include/fir_cuda.h and the
  sm_100a kernels (nvcc, ``-gencode arch=compute_100a,code=sm_100a``).
* ``fir_b200/lib/libfir.so`` and ``fir_b200/bin/FIR_*`` -- the C++ drop-in layer
  (FIR's headers and executables over the C ABI), when its sources exist.

All float and double arithmetic is compiled without FMA contraction
(``--fmad=false`` for device code, ``-ffp-contract=off`` for host code): the
kernels round every operation the way FIR's x86-64 build does.

Run ``python -m fir_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
BIN_DIR = os.path.join(HERE, "bin")
CUDA_LIB = os.path.join(LIB_DIR, "libfir_cuda.so")
HOST_LIB = os.path.join(LIB_DIR, "libfir.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"  # the image's $CXX wrapper lacks OpenMP specs

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--fmad=false",
    "-Xcompiler",
    "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-ccbin",
    CXX,
]


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_cuda(force: bool = False, verbose: bool = True, extra=()) -> str:
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = srcs + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps.append(os.path.join(ROOT, "include", "fir_cuda.h"))
    if force or _newer(CUDA_LIB, deps):
        os.makedirs(LIB_DIR, exist_ok=True)
        tmp = CUDA_LIB + ".tmp"
        _run([NVCC] + ARCH + NVCC_FLAGS + list(extra) + ["-shared", "-o", tmp] + srcs, verbose)
        os.replace(tmp, CUDA_LIB)
    return CUDA_LIB


def build_host(force: bool = False, verbose: bool = True) -> None:
    """C++ drop-in layer: libfir.so + FIR_ForwardProj / FIR_BackProj / FIR_OSEM."""
    host_dir = os.path.join(CSRC, "host")
    srcs = sorted(glob.glob(os.path.join(host_dir, "*.cc")))
    if not srcs:
        return
    hdrs = glob.glob(os.path.join(host_dir, "include", "*"))
    flags = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-I", os.path.join(host_dir, "include"),
             "-I", os.path.join(ROOT, "include")]
    os.makedirs(LIB_DIR, exist_ok=True)
    if force or _newer(HOST_LIB, srcs + hdrs + [CUDA_LIB]):
        _run([CXX] + flags + ["-shared", "-o", HOST_LIB] + srcs +
             ["-L", LIB_DIR, "-lfir_cuda", "-Wl,-rpath,$ORIGIN"], verbose)
    bins = sorted(glob.glob(os.path.join(CSRC, "bin", "*.cc")))
    os.makedirs(BIN_DIR, exist_ok=True)
    for b in bins:
        name = "FIR_" + os.path.splitext(os.path.basename(b))[0]
        out = os.path.join(BIN_DIR, name)
        if force or _newer(out, [b, HOST_LIB] + hdrs):
            _run([CXX] + flags + ["-o", out, b, "-L", LIB_DIR, "-lfir", "-lfir_cuda",
                                  "-Wl,-rpath,$ORIGIN/../lib"], verbose)


def build(force: bool = False, verbose: bool = True) -> None:
    build_cuda(force, verbose)
    build_host(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
