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

SOURCES = ["chaste_gpu.cu", "partition.cu", "noalloc.cu", "batch.cu", "runs.cu", "cable.cu", "selftest.cu",
           "host/assemble.cpp"]


def _deps():
    """Every source and header under csrc/ plus the public header: a change to any
    of them rebuilds the library."""
    out = ["../../include/chaste_gpu.h"]
    for root, _, files in os.walk(CSRC):
        for f in files:
            if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                out.append(os.path.relpath(os.path.join(root, f), CSRC))
    return sorted(out)


DEPS = _deps()


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
    """Compile libchastegpu.so for sm_100a when it is missing or older than its sources.
    The translation units compile in parallel (one nvcc each), then link."""
    import concurrent.futures

    os.makedirs(LIB_DIR, exist_ok=True)
    out = os.path.join(LIB_DIR, "libchastegpu.so")
    if force or _stale(out, DEPS):
        obj_dir = os.path.join(LIB_DIR, "obj")
        os.makedirs(obj_dir, exist_ok=True)
        compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

        def compile_one(src):
            obj = os.path.join(obj_dir, src.replace("/", "_") + ".o")
            cmd = [nvcc()] + ARCH + compile_flags + ["-c", "-o", obj, os.path.join(CSRC, src)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True, cwd=CSRC)
            return obj

        with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            objs = list(ex.map(compile_one, SOURCES))
        cmd = [nvcc()] + ARCH + ["-shared", "-o", out] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    return out


if __name__ == "__main__":
    print(build_native(force=True, verbose=True))
