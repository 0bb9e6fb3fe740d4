"""Build the in-tree CUDA library ``tmixer_b200/libtmx.so`` (sm_100a) and the
C++ driver ``tmixer_b200/tmx_run``.

nvcc cross-compiles without a GPU.  ``--fmad=false`` keeps every multiply and
add separately rounded (the reference is built for x86-64 without FMA
contraction); the kernels fuse only where they say so with ``__fma_rn``.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libtmx.so")
RUN = os.path.join(PKG, "tmx_run")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]
# per-source contraction: the FP64 kernels and the host code keep every
# operation separately rounded; the reduced-precision kernels may fuse
SOURCES = {"tmx_kernels.cu": ["--fmad=false"], "tmx_api.cu": ["--fmad=false"], "tmx_kernels_lp.cu": ["--fmad=true"],
           "tmx_batch.cu": ["--fmad=false"], "tmx_probe.cu": []}
# host-only C++ sources of the library (no device code)
CXX_SOURCES = {"tmx_serve.cpp": [], "tmx_writers.cpp": []}
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall"]
OBJDIR = os.path.join(PKG, "_build")


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "tmx.h"))
    os.makedirs(OBJDIR, exist_ok=True)
    objs, jobs = [], []
    for src, flags in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJDIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [_nvcc()] + NVCC_FLAGS + flags + ARCH + ["-c", "-o", obj, path]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            jobs.append((cmd, subprocess.Popen(cmd)))
    for src, flags in CXX_SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJDIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = ["g++"] + CXX_FLAGS + flags + ["-c", "-o", obj, path]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            jobs.append((cmd, subprocess.Popen(cmd)))
    for cmd, proc in jobs:
        if proc.wait() != 0:
            raise subprocess.CalledProcessError(proc.returncode, cmd)
    if force or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", tmp] + objs
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    drv = os.path.join(CSRC, "tmx_run.cpp")
    if os.path.exists(drv) and (force or _stale(RUN, [drv, LIB])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), drv, "-o", RUN,
               "-L", PKG, "-ltmx", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
