"""Build libgamgpu.so (the C-ABI library of the GAMERA step) in-tree with nvcc for sm_100a."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgamgpu.so")
SOURCES = ["gam_capi.cu", "gam_step.cu", "gam_flux.cu", "gam_efield.cu", "gam_init.cu", "gam_ring.cu",
           "gam_noalloc.cu", "gam_flux_f32.cu", "gam_efield_f32.cu", "gam_io.cu", "gam_tiles.cu",
           "gam_net.cu", "gam_closure.cu", "gam_msph.cu"]
# The FP32-flux kernels use approximate single-precision division and square root (their error budget is
# the FP32 path's 1e-5 L1 bound); every other unit keeps IEEE arithmetic. These flags touch
# single-precision operations only.
FAST_F32 = {"gam_flux_f32.cu", "gam_efield_f32.cu"}
FAST_F32_FLAGS = ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
OBJDIR = os.path.join(HERE, "_build")
DRIVER_SRC = os.path.join(HERE, "driver", "gamera_gpu_x.cpp")
DRIVER = os.path.join(HERE, "driver", "gamera_gpu_x")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(DRIVER_SRC)
    if not os.path.exists(DRIVER):
        return True
    deps.append(os.path.join(ROOT, "include", "gamgpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    common = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I", CSRC, "-I", os.path.join(ROOT, "include")]
    if verbose:
        common.insert(1, "-Xptxas=-v")
    procs, objs = [], []
    for src in SOURCES:   # one nvcc per unit, in parallel
        obj = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        cmd = common + (FAST_F32_FLAGS if src in FAST_F32 else []) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [src for src, pr in procs if pr.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc " + " ".join(failed))
    subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objs], check=True)
    build_driver()
    return LIB


def build_driver() -> str:
    """The C++ host driver over the C ABI (links libgamgpu.so from the package directory)."""
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), DRIVER_SRC, "-o", DRIVER,
           "-L", HERE, "-lgamgpu", "-Wl,-rpath,$ORIGIN/.."]
    subprocess.run(cmd, check=True)
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
