"""Build recipe of libjellyfih.so: nvcc, sm_100a only, in-tree output.

    python -m jellyfih_b200.build [--verbose]

The library is a plain C-ABI shared object (include/jellyfih.h) with the CUDA
runtime linked statically; it is loaded with ctypes by jellyfih_b200._lib.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libjellyfih.so")
SOURCES = ["jf_capi.cu", "jf_plain.cu", "jf_batched.cu", "jf_noalloc.cu", "jf_grad.cu", "jf_render.cu", "jf_tank.cu"]
HEADERS = ["jf_device.cuh", "jf_device64.cuh", "jf_engine.h", "jf_dual.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(REPO, "include", "jellyfih.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    # FMA contraction stays on; the rounding-sensitive P2G chain is written with
    # separately rounded intrinsics in jf_device.cuh.
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-I", os.path.join(REPO, "include"), "-o", LIB + ".tmp"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
