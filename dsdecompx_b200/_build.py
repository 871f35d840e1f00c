"""Build recipe of the in-tree native library (no JIT cache, no pip install).

``build()`` compiles every CUDA source under ``csrc/`` for sm_100a into
``_lib/libdsx.so`` (the C ABI of ``include/dsx.h`` plus the C++ drop-in of
``include/dsdecompx.hpp``) and the C++ parity programs under ``tests/cpp``.
``nvcc`` cross-compiles without a GPU.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libdsx.so")
INCLUDE = os.path.join(ROOT, "include")
# header-only single-process <mpi.h> for the C++ drop-in where no MPI exists
MPI_STUB = os.path.join(INCLUDE, "dsx_mpi_stub")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the FP64 wrap / shift / sum expressions must round like the
# reference's (no contraction into FMA).
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-Wall", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build dsdecompx_b200")
    return path


def sources() -> List[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale(target: str, deps: List[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) \
        + glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.hpp"))
    if force or _stale(LIB, deps):
        cmd = [nvcc()] + NVCC_FLAGS + ["-shared", "-I" + INCLUDE, "-I" + MPI_STUB, "-I" + CSRC,
                                       "-o", LIB] + sources() + ["-lcuda"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


WORKLOAD_LIB = os.path.join(LIBDIR, "libdsx_workload.so")
WORKLOAD_SRC = os.path.join(PKG, "workload", "workload.cu")


def build_workload(force: bool = False, verbose: bool = False) -> str:
    """Benchmark-harness kernels (synthetic drift and ghost forces)."""
    os.makedirs(LIBDIR, exist_ok=True)
    if force or _stale(WORKLOAD_LIB, [WORKLOAD_SRC, os.path.join(INCLUDE, "dsx.h")]):
        cmd = [nvcc()] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                                 "-I" + INCLUDE, "-o", WORKLOAD_LIB, WORKLOAD_SRC]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return WORKLOAD_LIB


def build_cpp_tests(force: bool = False, verbose: bool = False) -> List[str]:
    """C++ programs under tests/cpp that exercise the drop-in API like the
    reference's own sanity checks."""
    out = []
    for src in sorted(glob.glob(os.path.join(ROOT, "tests", "cpp", "*.cpp")) +
                      glob.glob(os.path.join(ROOT, "tests", "cpp", "*.cu"))):
        exe = os.path.join(LIBDIR, os.path.splitext(os.path.basename(src))[0])
        if force or _stale(exe, [src, LIB]):
            cmd = [nvcc()] + ARCH + ["-O2", "-std=c++17", "-I" + INCLUDE, "-I" + MPI_STUB, "-o", exe, src,
                                     "-L" + LIBDIR, "-ldsx", "-Xlinker", "-rpath=" + LIBDIR]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        out.append(exe)
    return out


def build(force: bool = False, verbose: bool = False) -> None:
    build_library(force=force, verbose=verbose)
    build_workload(force=force, verbose=verbose)
    build_cpp_tests(force=force, verbose=verbose)
