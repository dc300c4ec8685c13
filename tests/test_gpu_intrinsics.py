"""The FP32 XY decisions bound __sincosf's error by a constant measured on
sm_100a (kSincosfAbsErr in csrc/umc_math64.cuh).  This re-measures it
exhaustively on the GPU at hand (tests/cpp/sincosf_bound.cu, every FP32
angle with |x| <= 8) and fails if the hardware's error exceeds the constant."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "universal_classical_montecarlo_b200", "csrc")
SRC = os.path.join(ROOT, "tests", "cpp", "sincosf_bound.cu")
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")


@pytest.mark.gpu
def test_sincosf_error_within_the_decision_bound(tmp_path):
    if not os.path.isfile(NVCC):
        pytest.skip("nvcc not available")
    out = str(tmp_path / "sincosf_bound")
    cmd = [NVCC, "-std=c++20", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", f"-I{CSRC}", SRC, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    print(r.stdout)
    assert r.stdout.strip().splitlines()[-1] == "ok", r.stdout
