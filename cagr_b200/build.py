"""Builds libcagr_b200.so in-tree with nvcc for sm_100a.

    python -m cagr_b200.build          # or cagr_b200.build.build()

The library is plain C ABI (include/cagr.h): no torch headers, static CUDA
runtime, loaded from Python with ctypes.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libcagr_b200.so")
BIN_DIR = os.path.join(PKG, "bin")
# the GaussRecon driver on the C ABI (cli/main_gaussrecon.cpp), linked to the library
GAUSSRECON_PATH = os.path.join(BIN_DIR, "main_GaussReconCUDA")
SOURCES = ["capi.cu", "tree_build.cu", "moments.cu", "traverse.cu", "diagnostics.cu",
           "noalloc.cu", "mcubes.cu", "memory.cu", "interp.cu"]
HEADERS = ["common.cuh", "internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "cagr.h"))
    deps.append(os.path.join(PKG, "cli", "main_gaussrecon.cpp"))
    if not os.path.exists(GAUSSRECON_PATH):
        return True
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu into the shared library (skipped when up to date)."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB_PATH)
    build_gaussrecon(verbose)
    return LIB_PATH


def build_gaussrecon(verbose: bool = False) -> str:
    """The C++ main_GaussReconCUDA, linked to libcagr_b200.so (found next to it
    through its rpath: ../lib)."""
    os.makedirs(BIN_DIR, exist_ok=True)
    tmp = GAUSSRECON_PATH + ".tmp"
    cmd = [nvcc(), *ARCH, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           os.path.join(PKG, "cli", "main_gaussrecon.cpp"), "-o", tmp, "-L", LIB_DIR, "-lcagr_b200",
           "-Xlinker", "-rpath=$ORIGIN/../lib"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, GAUSSRECON_PATH)
    return GAUSSRECON_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
