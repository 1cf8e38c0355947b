"""Build the sm_100a shared library libgz_b200.so in-tree with nvcc.

    python -m graphzeppelin_b200.build [--force] [--verbose]

The library is the product: the CUDA kernels plus the C ABI declared in include/gz_b200.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libgz_b200.so")
GEN_LIB = os.path.join(PKG, "libgz_gen.so")
SOURCES = ["gz_kernels.cu", "gz_planes.cu", "gz_capi.cu", "gz_noalloc.cu", "gz_batch.cu"]
HEADERS = ["gz_device.cuh", "gz_kernels.cuh", "gz_common.cuh", "gz_ingest_plan.h", os.path.join("..", "..", "include", "gz_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libgz_b200.so")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_gen(force: bool = False) -> str:
    """Host-side stream generator (plain C + OpenMP)."""
    src = os.path.join(CSRC, "gz_gen.c")
    if not force and os.path.exists(GEN_LIB) and os.path.getmtime(GEN_LIB) >= os.path.getmtime(src):
        return GEN_LIB
    tmp = GEN_LIB + f".tmp{os.getpid()}"
    cc = shutil.which("gcc") or "cc"
    res = subprocess.run([cc, "-O3", "-std=c11", "-fopenmp", "-fPIC", "-shared",
                          "-fvisibility=hidden", "-o", tmp, src, "-lm"], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("gcc failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, GEN_LIB)
    return GEN_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    build_gen(force)
    if not force and not _stale():
        return LIB
    tmp = LIB + f".tmp{os.getpid()}"
    cmd = [nvcc_path(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-shared", "-o", tmp]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
