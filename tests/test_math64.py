"""FP64 sine and cosine of the deferred accept decisions (csrc/umc_math64.cuh),
checked on the CPU against the long-double library (tests/cpp/sincos_check.cu,
built by nvcc; no GPU needed): within 4 units of 2^-53 on every FP32 angle
sample in [-8, 8], next to the quadrant edges, and on FP64 values up to 2^19."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "universal_classical_montecarlo_b200", "csrc")
SRC = os.path.join(ROOT, "tests", "cpp", "sincos_check.cu")
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")


def test_sincos_cw64_accuracy(tmp_path):
    if not os.path.isfile(NVCC):
        pytest.skip("nvcc not available")
    out = str(tmp_path / "sincos_check")
    cmd = [NVCC, "-std=c++20", "-O2", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets", f"-I{CSRC}", SRC,
           "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().splitlines()[-1] == "ok", r.stdout
