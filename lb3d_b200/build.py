"""Builds the sm_100a CUDA library lb3d_b200/_lib/liblb3dc.so in-tree.

nvcc cross-compiles for sm_100a without a GPU.  The FP64 drop-in kernels
(fp64_path.cu) and the host-side C-ABI are compiled without FMA contraction
(--fmad=false, -ffp-contract=off) so that they reproduce the CPU
restatement bit for bit.  The FP32 kernels are compiled the same way and
spell out each fused multiply-add they want (fmaf, paired __ffma2_rn), so
every FP32 strategy rounds identically.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liblb3dc.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
               "-ffp-contract=off", "--expt-relaxed-constexpr"]
SOURCES = {
    # source: extra flags
    "fp64_path.cu": ["--fmad=false"],
    "reduce.cu": ["--fmad=false"],
    "capi.cu": ["--fmad=false"],
    # the FP32 kernels spell out every fused multiply-add (fmaf, paired
    # __ffma2_rn), so all strategies round identically
    "fp32_path.cu": ["--fmad=false"],
    "ensemble.cu": [],
    "noalloc.cu": [],
}
CXX_SOURCES = {"xdr.cpp": []}


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "lb3dc.h"))
    return hs


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers() + [__file__])


def build(verbose=False, force=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    objs, cmds = [], []
    for src, extra in SOURCES.items():
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, path):
            cmds.append([nvcc] + ARCH + NVCC_COMMON + extra + ["-c", path, "-o", obj])
    for src, extra in CXX_SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, path):
            cmds.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off"] + extra + ["-c", path, "-o", obj])
    # the translation units compile independently: run them side by side
    from concurrent.futures import ThreadPoolExecutor
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), flush=True)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(subprocess.check_call, cmd) for cmd in cmds]:
            f.result()
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
