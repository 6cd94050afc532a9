"""Builds libmercury_mhd.so in-tree with nvcc for sm_100a.

The FP64 parity path must reproduce the reference's x86-64 operation order,
so every translation unit is compiled with --fmad=false (no FMA contraction)
and IEEE division and square root, except the FP32 instantiation of the step
kernels (mixed precision), which is compiled separately with FMA contraction
and approximate division and square root."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmercury_mhd.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
EXACT = ["--fmad=false"]
FAST32 = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-DMHD_KERNELS_F32=1"]
# (source, object, flags)
UNITS = [
    ("mhd_kernels.cu", "mhd_kernels_f64.o", EXACT),
    ("mhd_kernels.cu", "mhd_kernels_f32.o", FAST32),
    ("mhd_ctx.cu", "mhd_ctx.o", EXACT),
    ("mhd_topology.cpp", "mhd_topology.o", EXACT),
    ("mhd_multiblock.cpp", "mhd_multiblock.o", EXACT),
    ("mhd_noalloc.cu", "mhd_noalloc.o", EXACT),
    ("mhd_host_setup.cpp", "mhd_host_setup.o", EXACT),
    ("mhd_restart.cpp", "mhd_restart.o", EXACT),
    ("mhd_tecplot.cpp", "mhd_tecplot.o", EXACT),
    ("mhd_geometry.cu", "mhd_geometry.o", EXACT),
]
SOURCES = sorted({u[0] for u in UNITS})


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "mercury_mhd.h"),
                                                                 os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    common = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
              "-I" + os.path.join(ROOT, "include")]
    procs = []
    objs = []
    for src, obj, flags in UNITS:
        out = os.path.join(OBJ, obj)
        cmd = [nvcc, *common, *flags, "-c", os.path.join(CSRC, src), "-o", out]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append(subprocess.Popen(cmd))
        objs.append(out)
    if any(p.wait() != 0 for p in procs):
        raise subprocess.CalledProcessError(1, "nvcc")
    link = [nvcc, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.check_call(link)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
