"""Build the B200 DEM library (lib/libesys_dem_b200.so) with nvcc for sm_100a.

The FP64 kernels are compiled with --fmad=false so that every + - * / sqrt is
rounded like the reference's x86-64 double arithmetic (no fused multiply-add).
Run: python esys-particle_b200/build.py  (idempotent; rebuilds when sources change).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libesys_dem_b200.so")
SOURCES = ["dem_kernels.cu", "dem_sim.cu", "dem_noalloc.cu", "packing.cpp"]
HEADERS = ["dem_device.cuh", "dem_kernels.h", "dem_laws.cuh", "dem_math.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("esys_dem.h", "esys_geometry.h")]
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC", "-shared",
           "-o", LIB + ".tmp"] + [os.path.join(SRC, f) for f in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
