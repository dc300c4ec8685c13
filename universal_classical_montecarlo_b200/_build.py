"""Builds libumc_b200.so in-tree: nvcc for the sm_100a kernels, g++ for host code.

Usage: ``python universal_classical_montecarlo_b200/_build.py`` (also called by
``__graft_entry__.build()``).  Objects go to ``_build/`` beside this file and
the shared library to the package directory, so the built artefact travels
with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libumc_b200.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", f"-I{INCLUDE}"]
CXX_FLAGS = ["-std=c++23", "-O2", "-fPIC", "-Wall", "-Wextra", f"-I{INCLUDE}", f"-I{CUDA_HOME}/include"]

CU_SOURCES = ["umc_chain.cu", "umc_gauge.cu", "umc_batch.cu", "umc_learn.cu", "umc_noalloc.cu", "umc_slab.cu", "umc_gslab.cu"]
CXX_SOURCES = ["umc_tables.cpp", "umc_stats.cpp"]


def _sources():
    cu = [s for s in CU_SOURCES if os.path.isfile(os.path.join(CSRC, s))]
    cxx = [s for s in CXX_SOURCES if os.path.isfile(os.path.join(CSRC, s))]
    return cu, cxx


def _deps():
    shared = [os.path.join(INCLUDE, "umc", f) for f in os.listdir(os.path.join(INCLUDE, "umc")) if f.endswith(".cuh")]
    # this file too: a change of flags rebuilds
    return ([os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "umc_b200.h")] + shared
            + [os.path.abspath(__file__)])


def _stale(obj: str, src: str) -> bool:
    if not os.path.isfile(obj):
        return True
    t = os.path.getmtime(obj)
    # headers are shared: any newer file under csrc/ rebuilds everything
    return any(os.path.getmtime(d) > t for d in _deps() + [src])


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, jobs: int | None = None) -> str:
    if not os.path.isfile(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    cu, cxx = _sources()
    steps = []
    objs = []
    for s in cu:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if _stale(obj, src):
            steps.append([NVCC, *ARCH, *NVCC_FLAGS, "-Xptxas", "-v", "-c", src, "-o", obj])
    for s in cxx:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if _stale(obj, src):
            steps.append(["g++", *CXX_FLAGS, "-c", src, "-o", obj])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for out in ex.map(_run, steps):
            logs.append(out)
    if steps or not os.path.isfile(LIB):
        tmp = LIB + ".tmp"
        _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
        os.replace(tmp, LIB)
    if verbose:
        for l in logs:
            sys.stdout.write(l)
    return LIB


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    if os.path.exists(LIB):
        os.remove(LIB)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
