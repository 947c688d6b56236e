"""Build the sm_100a library in-tree: simple-cpsd_b200/lib/libcpsd_b200.so.

nvcc cross-compiles without a GPU, so this runs anywhere the CUDA toolkit is
installed.  The output stays in the source tree (not site-packages) so that
it travels with the repository.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))  # simple-cpsd_b200/
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(REPO_ROOT, "include")
LIBDIR = os.path.join(PKG_ROOT, "lib")
LIB = os.path.join(LIBDIR, "libcpsd_b200.so")

SOURCES = ["engine.cu", "capi.cu"]
HEADERS = ["common.cuh", "dropin.h", "fft.cuh", "host_pool.h", "kernels.cuh", "mlp.cuh", "pipeline.cuh", "tc_gemm.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-shared",
]


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "cpsd_b200.h"))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs() if os.path.exists(f))


def build_library(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-I" + INCLUDE, "-I" + CSRC]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    cmd += ["-o", LIB + ".tmp", "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
