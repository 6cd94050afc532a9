"""Builds libmercury_mhd.so in-tree with nvcc for sm_100a.

The FP64 parity path must reproduce the reference's x86-64 operation order,
so the whole library is compiled with --fmad=false (no FMA contraction);
division and square root stay IEEE-rounded (nvcc defaults)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmercury_mhd.so")
SOURCES = ["mhd_kernels.cu", "mhd_ctx.cu", "mhd_topology.cpp", "mhd_noalloc.cu", "mhd_host_setup.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "mercury_mhd.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "--fmad=false", "-std=c++17", "--extended-lambda", "--threads", "0", "-Xcompiler", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "include"), "-o", LIB + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES], "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
