"""Build recipe for librisgraph_b200.so (sm_100a) and its host tools.

The shared library is built in-tree (risgraph_b200/librisgraph_b200.so) with
explicit nvcc commands, so the same file is what loads on a GPU machine.
Run `python -m risgraph_b200.build` or call build().
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "librisgraph_b200.so")
BIN = os.path.join(PKG, "bin")
DRIVER = os.path.join(BIN, "rg_driver")
# the reference's command-line drivers, all served by one binary (argv[0] picks)
DRIVER_NAMES = [a + m for a in ("bfs", "sssp", "sswp", "wcc") for m in ("", "_inc", "_inc_batch", "_inc_rt")]
# the reference's text -> binary converters, one binary likewise
CONVERT = os.path.join(BIN, "rg_convert")
CONVERT_NAMES = ["convert_to_binary", "convert_to_binary_random", "convert_to_binary_timestamp"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"
HOST_CC = "/usr/bin/gcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-ccbin", HOST_CXX, "-Xcompiler", "-fPIC",
                  "-I" + INCLUDE, "-I" + CSRC, "--expt-relaxed-constexpr"]

CU_SOURCES = ["rg_api.cu", "rg_storage.cu", "rg_tree.cu", "rg_static.cu", "rg_serve.cu", "rg_history.cu", "rg_autotune.cu"]
C_SOURCES = ["rg_gen.c"]
CXX_SOURCES = ["rg_front.cpp"]
HEADERS = ["rg_internal.cuh", "rg_storage_dev.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and r.stderr.strip():
        sys.stderr.write(r.stderr)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "risgraph_b200.h"),
                                                       os.path.join(INCLUDE, "rg_gen.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if force or _newer(o, [s] + hdrs):
            _run([NVCC] + NVFLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cpp", ".o"))
        if force or _newer(o, [s] + hdrs):
            _run([HOST_CXX, "-O2", "-fPIC", "-std=c++17", "-Wall", "-I" + INCLUDE, "-c", s, "-o", o], verbose)
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".c", ".o"))
        if force or _newer(o, [s] + hdrs):
            _run([HOST_CC, "-O3", "-fPIC", "-fopenmp", "-std=c11", "-I" + INCLUDE, "-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-ccbin", HOST_CXX, "-shared", "-o", LIB] + objs +
             ["-Xcompiler", "-fopenmp", "-lgomp", "-cudart", "static"], verbose)
    build_drivers(verbose, force)
    return LIB


def build_drivers(verbose: bool = False, force: bool = False) -> str:
    """risgraph_b200/bin/rg_driver and its links bfs, sssp_inc, wcc_inc_rt, ..."""
    os.makedirs(BIN, exist_ok=True)
    src = os.path.join(PKG, "cli", "rg_driver.cpp")
    if force or _newer(DRIVER, [src, LIB, os.path.join(INCLUDE, "risgraph_b200.h")]):
        _run([HOST_CXX, "-std=c++17", "-O2", "-fopenmp", "-I" + INCLUDE, src, "-L" + PKG, "-lrisgraph_b200",
              "-Wl,-rpath,$ORIGIN/..", "-o", DRIVER], verbose)
    src = os.path.join(PKG, "cli", "rg_convert.cpp")
    if force or _newer(CONVERT, [src, LIB]):
        _run([HOST_CXX, "-std=c++17", "-O2", "-I" + INCLUDE, src, "-L" + PKG, "-lrisgraph_b200",
              "-Wl,-rpath,$ORIGIN/..", "-o", CONVERT], verbose)
    for target, names in (("rg_driver", DRIVER_NAMES), ("rg_convert", CONVERT_NAMES)):
        for name in names:
            link = os.path.join(BIN, name)
            if not os.path.islink(link):
                if os.path.exists(link):
                    os.remove(link)
                os.symlink(target, link)
    return DRIVER


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
