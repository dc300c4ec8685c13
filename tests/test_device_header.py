"""Host-side arithmetic of include/umc/device.cuh, checked on the CPU
(tests/cpp/device_host_check.cu, built by nvcc; no GPU needed): the
multiply-high division, RegularLattice's colour-major numbering and computed
neighbours against a direct construction, the checkerboard colouring and its
refusals, Classes::from_colours, and the device Rng against a sequential
reference Pcg32 with the keyed seed."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "universal_classical_montecarlo_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "device_host_check.cu")
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")


def test_device_header_host_arithmetic(tmp_path, umc):
    if not os.path.isfile(NVCC):
        pytest.skip("nvcc not available")
    out = str(tmp_path / "device_host_check")
    cmd = [NVCC, "-std=c++20", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "--expt-relaxed-constexpr",
           "-diag-suppress", "177,20011", f"-I{os.path.join(ROOT, 'include')}", SRC, f"-L{PKG}", "-lumc_b200",
           "-Xlinker", f"-rpath,{PKG}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
