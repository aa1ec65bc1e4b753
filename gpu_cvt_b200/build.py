"""Build libgpucvt.so (the sm_100a kernels + C ABI) in-tree with nvcc.

    python -m gpu_cvt_b200.build          # build if sources changed
    python -m gpu_cvt_b200.build --force  # rebuild

-fmad=false pins the rounding of every FP32/FP64 expression (explicit
fma() calls are the only fused operations), which is what lets the kernels
agree bit-for-bit with a CPU restatement that follows the same operation order.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgpucvt.so")
NVCC = os.environ.get("NVCC", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  [os.path.join(ROOT, "include", "gpu_cvt.h")])


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [NVCC] + ARCH + FLAGS + (extra or []) + ["-o", LIB, os.path.join(CSRC, "cvt_capi.cu")]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
