"""Builds libexogcm.so (the CUDA engine and its C ABI) in-tree for sm_100a."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libexogcm.so")
SOURCES = ["engine.cu", "transforms.cu", "legendre.cu", "legendre_tc.cu", "fft.cu", "spectral_grid.cu", "dynamics.cu",
           "physics.cu", "noalloc.cu", "setup.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
# Column physics uses the GPU's fast arithmetic: division and square root to
# 2 ulp (WGSL allows its division 2.5 ulp), exp/log/pow from the
# special-function unit (relative error about 1e-6), denormals flushed to
# zero. These fits (absorptivities, saturation, cloud optics) carry
# empirical coefficients of 3-4 digits, and the per-column kernels are
# bound by their instruction count, so the accurate library routines would
# cost speed and add nothing the FP64 comparison can see.
# The grid-point dynamics kernels divide to 2 ulp as well (-prec-div=false):
# elementwise kernels such as physics_out spent most of their issue slots in
# the IEEE division sequence.
FILE_FLAGS = {"physics.cu": ["-use_fast_math"], "dynamics.cu": ["-prec-div=false"]}


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    for name in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, name)) > built:
            return True
    header = os.path.join(HERE, "..", "include", "exogcm.h")
    return os.path.getmtime(header) > built


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objects = []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [NVCC, *FLAGS, *FILE_FLAGS.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-c",
                   os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objects.append(obj)
    # cudart links statically (nvcc's default), so the library loads on a
    # host without a CUDA runtime install and fails only at its first device call.
    subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objects],
                   check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
