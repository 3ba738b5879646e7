"""Builds the in-tree shared libraries of the package with nvcc/g++.

libexcl_gpu.so   the product: C ABI (include/excl_gpu.h) + sm_100a kernels
libexcl_synth.so seeded synthetic workloads for tests and benchmarks

Device code is compiled for sm_100a only. Host code that must reproduce the
reference's floating-point arithmetic (codec.cpp: regression fits) is compiled
with -ffp-contract=off and no -march flag.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-ffp-contract=off",
              "--expt-relaxed-constexpr", f"-I{INCLUDE}"]
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-pthread", f"-I{INCLUDE}"]

GPU_SOURCES = ["codec.cpp", "kernels.cu", "decode.cu", "runtime.cu", "learned_train.cu", "noalloc.cu",
               "serve.cu", "refformat.cpp", "build_gpu.cu"]
GPU_HEADERS = ["excl_internal.h", "excl_device.cuh", "kernels.h", "runtime.h", "batch_phases.cuh"]
SYNTH_SOURCES = ["synth.cpp"]

LIB_GPU = os.path.join(PKG, "libexcl_gpu.so")
LIB_SYNTH = os.path.join(PKG, "libexcl_synth.so")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def _compile(src: str, verbose: bool, extra_deps: list[str]) -> str:
    os.makedirs(BUILD, exist_ok=True)
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    deps = [path, os.path.join(INCLUDE, "excl_gpu.h"), *extra_deps]
    if _newer(obj, deps):
        return obj
    if src.endswith(".cu"):
        _run([NVCC, *NVCC_FLAGS, "-c", path, "-o", obj], verbose)
    else:
        _run(["g++", *CXX_FLAGS, "-c", path, "-o", obj], verbose)
    return obj


def build(verbose: bool = False) -> None:
    hdrs = [os.path.join(CSRC, h) for h in GPU_HEADERS]
    objs = [_compile(s, verbose, hdrs) for s in GPU_SOURCES]
    if not _newer(LIB_GPU, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB_GPU, *objs, "-lpthread"], verbose)
    sobjs = [_compile(s, verbose, []) for s in SYNTH_SOURCES]
    if not _newer(LIB_SYNTH, sobjs):
        _run(["g++", "-shared", "-pthread", "-o", LIB_SYNTH, *sobjs], verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print("built", LIB_GPU, LIB_SYNTH)
