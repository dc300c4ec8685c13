"""Builds examples/device_models/_build/libumc_device_models.so from
user_models.cu: user-written models compiled by nvcc against
include/umc/device.cuh and linked to libumc_b200.so, the way a user of the
library builds theirs.  Called by ``__graft_entry__.build()``, and by the tests
and bench.py when the library is missing or older than its sources.

Usage: ``python examples/device_models/build_device_models.py``
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "universal_classical_montecarlo_b200")
SRC = os.path.join(HERE, "user_models.cu")
OUT = os.path.join(HERE, "_build", "libumc_device_models.so")
HEADERS = [os.path.join(ROOT, "include", "umc", f) for f in ("device.cuh", "keyed_pcg.cuh")] + [
    os.path.join(ROOT, "include", "umc_b200.h")]
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-diag-suppress", "177"]


def stale() -> bool:
    if not os.path.isfile(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in [SRC, *HEADERS])


def build() -> str:
    if not stale():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    tmp = OUT + ".tmp"
    cmd = [NVCC, *FLAGS, f"-I{os.path.join(ROOT, 'include')}", "-shared", SRC, "-o", tmp, f"-L{PKG}", "-lumc_b200",
           "-Xlinker", "-rpath,$ORIGIN/../../../universal_classical_montecarlo_b200"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("device model build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build())
