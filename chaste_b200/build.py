"""Build the sm_100a shared library libchastegpu.so in-tree (chaste_b200/lib/)."""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]

SOURCES = ["chaste_gpu.cu", "noalloc.cu", "batch.cu", "cable.cu", "selftest.cu", "host/assemble.cpp"]
DEPS = SOURCES + [
    "kernels/common.cuh", "kernels/ops.cuh", "kernels/cg.cuh", "kernels/cg_mixed.cuh",
    "kernels/ode.cuh", "kernels/batch.cuh", "kernels/cable.cuh", "kernels/svi.cuh", "kernels/output.cuh",
    "models/cellmodel_common.h", "models/lr91.h", "models/tt06.h",
    "host/assemble.h", "../../include/chaste_gpu.h",
]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(os.path.join(CSRC, d)) > t for d in deps)


def build_native(force=False, verbose=False):
    """Compile libchastegpu.so for sm_100a when it is missing or older than its sources."""
    os.makedirs(LIB_DIR, exist_ok=True)
    out = os.path.join(LIB_DIR, "libchastegpu.so")
    if force or _stale(out, DEPS):
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-o", out] + [os.path.join(CSRC, s) for s in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    return out


if __name__ == "__main__":
    print(build_native(force=True, verbose=True))
