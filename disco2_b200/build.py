"""Build libdisco_gpu.so in-tree (disco2_b200/_lib/).

Host C (gcc, -ffp-contract=off) + sm_100a CUDA (nvcc -gencode
arch=compute_100a,code=sm_100a -fmad=false), linked into one shared library
whose exported symbols are exactly the C ABI of include/disco_gpu.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libdisco_gpu.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CC = shutil.which("gcc") or "gcc"

C_SOURCES = ["dgpu_sim.c", "dgpu_ctx.c", "dgpu_diff.c", "dgpu_h5.c", "dgpu_io.c"]
CU_SOURCES = ["dgpu_kernels.cu", "dgpu_adjoint.cu", "dgpu_diag.cu"]
HEADERS = ["dgpu_internal.h", "dgpu_sim.h", "dgpu_ctx.h", "dgpu_h5.h", "dgpu_device.cuh", "dgpu_step.cuh", "dgpu_adjoint.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-fmad=false",
    "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
] + os.environ.get("DGPU_NVCC_EXTRA", "").split()
C_FLAGS = ["-O2", "-std=gnu99", "-fPIC", "-ffp-contract=off", "-Wall",
           "-Wno-unused-function", f"-I{CUDA_HOME}/include", f"-I{ROOT}/include"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile what changed; return the library path."""
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "disco_gpu.h")]
    objs = []
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + hdrs):
            # the exported C ABI functions get default visibility through the
            # version script below; everything else stays hidden
            _run([CC, *C_FLAGS, "-c", s, "-o", o], verbose)
        objs.append(o)
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + hdrs):
            _run([NVCC, *NVCC_FLAGS, "-c", s, "-o", o], verbose)
        objs.append(o)
    vs = os.path.join(OBJ, "exports.map")
    with open(vs, "w") as f:
        f.write("{ global: dgpu_*; local: *; };\n")
    if force or _stale(LIB, objs + [vs]):
        cxx = shutil.which("g++") or "g++"
        _run([cxx, "-shared", "-fPIC", "-o", LIB, *objs, f"-Wl,--version-script={vs}",
              f"-L{CUDA_HOME}/lib64", "-lcudart_static", "-lrt", "-ldl", "-lpthread"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
