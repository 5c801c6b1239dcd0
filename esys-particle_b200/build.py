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
# (source, FMA contraction): the FP64 path is built without FMA so that it rounds
# like the reference; the FP32-force instances use FMA.
SOURCES = [("dem_kernels.cu", False), ("dem_sim.cu", False), ("dem_noalloc.cu", False), ("dem_step_fp32.cu", True),
           ("dem_adjoint.cu", False), ("dem_batch.cu", False), ("dem_batch_fp32.cu", True),
           ("packing.cpp", False)]
HEADERS = ["dem_device.cuh", "dem_kernels.h", "dem_laws.cuh", "dem_laws_f32.cuh", "dem_math.cuh", "dem_common.cuh",
           "dem_step.cuh", "dem_tiled.cuh", "dem_adjoint.h", "dem_dual.cuh", "dem_batch.cuh", "dem_bond_vjp.cuh", "dem_pair_vjp.cuh"]
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
    deps = [os.path.join(SRC, f) for f, _ in SOURCES] + [os.path.join(SRC, f) for f in HEADERS]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("esys_dem.h", "esys_geometry.h")]
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    objs, procs = [], []
    for f, fma in SOURCES:
        obj = os.path.join(HERE, "_build", f + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", f"--fmad={'true' if fma else 'false'}",
               "-Xcompiler", "-fPIC", "-c", os.path.join(SRC, f), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((f, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for f, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {f}:\n" + out + err)
        if verbose:
            sys.stderr.write(err)
    r = subprocess.run([nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp"] + objs, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
