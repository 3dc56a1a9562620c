"""Builds the CUDA library in-tree: mac_b200/libmac_gpu.so (sm_100a).

-fmad=false keeps every FP64 expression in the reference's rounding order (no
fused multiply-add contraction), which is what makes the stencil, topology and
particle kernels bit-exact with the reference compiled by g++. It is given to
the translation units whose results are compared with the reference bit for
bit or hold the projection's FP64 arithmetic (topology, forces, extrapolation,
particles, the step, the pressure system); the multigrid preconditioner and
the network (CONTRACT_OK) only shape the CG iterates, whose FP64 residual
decides convergence, and are built with contraction on (the multigrid's first
kernel also applies the CG update x += alpha p, r -= alpha q, which then
rounds once per element instead of twice).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmac_gpu.so")
SOURCES = ["mac_ctx.cu", "mac_topology.cu", "mac_advect.cu", "mac_pressure.cu", "mac_mg.cu", "mac_step.cu", "mac_noalloc.cu", "mac_unet.cu",
           "mac_extrap_bc.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CONTRACT_OK = {"mac_mg.cu", "mac_unet.cu"}
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]


def flags_for(src: str) -> list:
    return FLAGS + (["-fmad=true"] if src in CONTRACT_OK else ["-fmad=false"])


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "mac_gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    jobs = []
    for s in SOURCES:
        o = os.path.join(objdir, s.replace(".cu", ".o"))
        cmd = [NVCC, *flags_for(s), "-c", os.path.join(CSRC, s), "-o", o]
        if verbose:
            print(" ".join(cmd))
        jobs.append((s, o, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    objs = []
    for s, o, p in jobs:
        _out, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{err}")
        objs.append(o)
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
