"""Build the sm_100a shared library libcosa_gpu.so in-tree with nvcc.

The library is plain C-ABI (include/cosa_gpu.h); it links only the CUDA
runtime, so any host language can bind it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libcosa_gpu.so")
SOURCES = ["cosa_gpu.cu", "io.cpp"]
HEADERS = ["common.cuh", "physics.cuh", "kernels_ref.cuh", "fused.cuh", "mg.cuh", "visc.cuh", "kom.cuh", "split.cuh", "faces.cuh",
           "moving.cuh", "force.cuh", "serve.cuh", "unsteady.cuh", "lsp.cuh"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def flags(verbose: bool = False):
    f = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++",
         "-I", os.path.join(ROOT, "include")]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", h) for h in ("cosa_gpu.h", "cosa_io.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [nvcc()] + flags(verbose) + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libcosa_gpu.so")
    if verbose:
        sys.stderr.write(r.stderr)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
    print(LIB)
