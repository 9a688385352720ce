"""Build recipe for libcfft_b200.so (sm_100a).

Host C++ (plan layer, space-group table, C ABI) is compiled with g++; the device
layer with nvcc for sm_100a; the shared library links the CUDA runtime statically
so it depends only on the driver.  The library is built in-tree next to this file.

    python crystallographicfft.jl_b200/build.py [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcfft_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-fPIC", "-std=c++17", "-Wall", "-Wno-unused-function"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH

HOST_SOURCES = ["spacegroups.cpp", "planner.cpp", "cabi.cpp"]
# The fast-path kernels are split by stage group and precision so nvcc runs in parallel.
DEVICE_SOURCES = ["exec.cu", "scft.cu", "sno.cu", "fast_planes_f32.cu", "fast_planes_f64.cu", "fast_other_f32.cu", "fast_other_f64.cu"]
HEADERS = ["cfft_internal.h", "exec.h", "device_common.cuh", "fast_api.h", "fast_kernels.cuh", "tma_planes.cuh", "scft.h", "sno.h",
           "fractal_tree.h"]


def _newer(src_paths, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False, extra_nvflags=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "cfft_b200.h")]
    objs, jobs = [], []
    for s in HOST_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if force or _newer([src] + headers, obj):
            jobs.append(["g++"] + CXXFLAGS + ["-I", INCLUDE, "-I", "/usr/local/cuda/include", "-c", src, "-o", obj])
        objs.append(obj)
    for s in DEVICE_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if force or _newer([src] + headers, obj):
            jobs.append([NVCC] + NVFLAGS + list(extra_nvflags or []) + ["-I", INCLUDE, "-c", src, "-o", obj])
        objs.append(obj)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j, verbose) for j in jobs]:
            f.result()
    if force or _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"], verbose)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else None
    print(build(force=a.force or a.ptxas_verbose, verbose=a.verbose, extra_nvflags=extra))
    sys.exit(0)
