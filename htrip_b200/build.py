"""Build recipe for the in-tree CUDA library ``htrip_b200/libhtrip_b200.so``.

nvcc cross-compiles for sm_100a only (no other architecture is emitted):
``-gencode arch=compute_100a,code=sm_100a``.  The library exposes the C ABI
declared in ``include/htrip_b200.h`` (and the C++ drop-in of
``include/htrip/``).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libhtrip_b200.so")
CPP_LIB = os.path.join(PKG, "libhtrip.so")   # C++20 htrip::MinPlusOracle drop-in
HOST = os.path.join(PKG, "host")
CXX = os.environ.get("CXX", "g++")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                              + glob.glob(os.path.join(ROOT, "include", "*.h"))
                              + glob.glob(os.path.join(ROOT, "include", "htrip", "*.hpp")))


def up_to_date(target, inputs):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(p) <= t for p in inputs)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Build libhtrip_b200.so (CUDA, sm_100a) and the C++ drop-in libhtrip.so."""
    lib = build_cuda(force, verbose, ptxas_info)
    build_cpp(force, verbose)
    return lib


def build_cpp(force: bool = False, verbose: bool = False) -> str:
    """libhtrip.so: the C++20 htrip::MinPlusOracle of include/htrip/, linked
    against libhtrip_b200.so (found next to it through an $ORIGIN rpath)."""
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    inputs = srcs + [LIB] + sorted(glob.glob(os.path.join(ROOT, "include", "htrip", "*.hpp")))
    if not force and up_to_date(CPP_LIB, inputs):
        return CPP_LIB
    cmd = [CXX, "-std=c++20", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include"),
           "-o", CPP_LIB, *srcs, "-L" + PKG, "-lhtrip_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return CPP_LIB


def build_cuda(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not ptxas_info and up_to_date(LIB, deps()):
        return LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0 or (ptxas_info and r.stderr):
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}")
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
