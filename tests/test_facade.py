"""The C++23 facade (include/umc/umc.hpp): it compiles warning-free with g++
-std=c++23 against the C ABI library (CPU), and the reference-style check
program passes on the GPU (tests/cpp/facade_check.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "universal_classical_montecarlo_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "facade_check.cpp")


def _build(out):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    cmd = [cxx, "-std=c++23", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{os.path.join(ROOT, 'include')}", SRC,
           f"-L{PKG}", "-lumc_b200", f"-Wl,-rpath,{PKG}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.fixture(scope="module")
def facade_binary(tmp_path_factory):
    return _build(str(tmp_path_factory.mktemp("facade") / "facade_check"))


def test_facade_compiles(facade_binary):
    assert os.path.isfile(facade_binary)


def test_facade_host_tables(facade_binary):
    """The host-side tables, PairGraph<double> with bond payloads included,
    behave as the reference's (tests/cpp/facade_check.cpp, `tables` mode)."""
    r = subprocess.run([facade_binary, "tables"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "tables: ok" in r.stdout


def test_facade_without_a_gpu_fails_loudly(facade_binary, umc):
    if umc.device_count() > 0:
        pytest.skip("a GPU is present")
    r = subprocess.run([facade_binary], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0  # std::runtime_error from the C ABI, no CPU fallback


@pytest.mark.gpu
def test_facade_reference_style_program(facade_binary):
    r = subprocess.run([facade_binary], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
