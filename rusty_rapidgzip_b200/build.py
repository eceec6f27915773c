"""Build the CUDA decoder library in-tree.

    python -m rusty_rapidgzip_b200.build          # librrg_gpu.so for sm_100a

nvcc compiles the single translation unit csrc/rrg_gpu.cu (kernels + host
orchestration + C ABI) for sm_100a and writes rusty_rapidgzip_b200/librrg_gpu.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
SOURCES = [os.path.join(CSRC, f) for f in ("rrg_gpu.cu", "rrg_kernels.cuh", "rrg_common.h")]
HEADER = os.path.join(ROOT, "include", "rrg_gpu.h")
OUT = os.path.join(HERE, "librrg_gpu.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    if force or stale(OUT, SOURCES + [HEADER]):
        cmd = [nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               "-o", OUT, os.path.join(CSRC, "rrg_gpu.cu")]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
