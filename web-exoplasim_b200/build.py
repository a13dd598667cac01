"""Builds libexogcm.so (the CUDA engine and its C ABI) in-tree for sm_100a."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libexogcm.so")
SOURCES = ["engine.cu", "transforms.cu", "legendre.cu", "legendre_tc.cu", "fft.cu", "spectral_grid.cu", "dynamics.cu",
           "physics.cu", "physics_flux.cu", "physics_storm.cu", "budget.cu", "noalloc.cu", "setup_device.cu", "setup.cpp", "server.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
# Column physics divides and takes square roots to 2 ulp (WGSL allows its
# division 2.5 ulp) and flushes denormals to zero; the longwave band fits take
# their base-2 logarithm and power from the special-function unit
# (EXOGCM_LWR_FAST_LOG2/EXP2); every other exp/log/pow is CUDA's accurate
# one. With -use_fast_math everywhere the longwave fluxes missed the
# reference's V3 gate (GPU error against FP64 within twice a sequential-f32
# build's) by 2-3x; these flags pass it at T21 L5/L10, T42 L10 and T63 L10.
# Where a tendency is a small difference of two states, the divisions are
# IEEE explicitly (__fdiv_rn): the implicit vertical diffusion and vdiff's
# tendencies, the large-scale condensation, spectrald's diffusion and mkdheat.
# IEEE division everywhere in the physics cost 45 % more step time at T42.
# The grid-point dynamics kernels divide to 2 ulp as well (-prec-div=false):
# elementwise kernels such as physics_out spent most of their issue slots in
# the IEEE division sequence.
PHYSICS_FLAGS = ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]
FILE_FLAGS = {"physics.cu": PHYSICS_FLAGS + ["-DEXOGCM_LWR_FAST_EXP2", "-DEXOGCM_LWR_FAST_LOG2"],
              "physics_flux.cu": PHYSICS_FLAGS, "dynamics.cu": ["-prec-div=false"],
              # The FP64 set-up kernels follow the host loops operation for
              # operation and must not contract a*b+c into one rounding.
              "setup_device.cu": ["-fmad=false"]}


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    for name in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, name)) > built:
            return True
    header = os.path.join(HERE, "..", "include", "exogcm.h")
    return os.path.getmtime(header) > built or os.path.getmtime(os.path.abspath(__file__)) > built


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
