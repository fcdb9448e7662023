"""Build libflowgpu.so (CUDA kernels for sm_100a + host C code) in-tree.

    python flow-solver_b200/build.py [--verbose]

The shared library lands in flow-solver_b200/lib/ so that it travels with
the source tree.  Kernels are compiled with --fmad=false: no multiply-add
contraction, which keeps the double-precision results identical to the
reference's host arithmetic.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(LIBDIR, "libflowgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "--fmad=false", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xptxas", "-v"]
HOST_SOURCES = ["host/quadrature.c", "host/svd.c", "host/curved.c", "host/prep.cpp"]
CUDA_SOURCES = ["flow_gpu.cu", "flow_serve.cu", "flow_output.cu"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return r.stdout + r.stderr


def build(verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I", os.path.join(CSRC, "host")]
    objs = []
    for src in HOST_SOURCES:
        obj = os.path.join(OBJDIR, os.path.splitext(os.path.basename(src))[0] + ".o")
        if src.endswith(".cpp"):
            cmd = ["g++", "-O2", "-fPIC", "-ffp-contract=off", "-std=c++17", "-Wall"]
        else:
            cmd = ["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-std=c99", "-D_DEFAULT_SOURCE",
                   "-Wall"]
        _run([*cmd, *inc, "-c", os.path.join(CSRC, src), "-o", obj], verbose)
        objs.append(obj)
    log = []
    for src in CUDA_SOURCES:
        obj = os.path.join(OBJDIR, os.path.basename(src).replace(".cu", ".o"))
        log.append(_run([nvcc(), *ARCH, *NVCC_FLAGS, *inc, "-c", os.path.join(CSRC, src),
                         "-o", obj], verbose))
        objs.append(obj)
    _run([nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], verbose)
    with open(os.path.join(OBJDIR, "ptxas.log"), "w") as f:
        f.write("\n".join(log))
    return LIB


if __name__ == "__main__":
    path = build(verbose="--verbose" in sys.argv)
    print("built", path)
