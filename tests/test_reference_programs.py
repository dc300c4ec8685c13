"""The reference's own test programs (test/*.cpp of the reference tree),
unchanged, built against the engine's facade through include/umc/compat: the
headers at the reference's include paths (driver.hpp, dof/sun.hpp, ...), each
declaring its reference header's names.  Every program but graph_check
compiles and links warning-free; plaquette_check and rotation_check check
host arithmetic only and pass here; model_check, su_check and u1_check run
chains, so without a GPU they stop with the engine's error (no CPU fallback),
and with one they must pass.  graph_check drives a host model type of its own
(IsingGraph), which the facade refuses at compile time with its message: such
a model runs through umc/device.cuh.  Skipped where the reference tree is
absent."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "universal_classical_montecarlo_b200")
INC = os.path.join(ROOT, "include")
HOST_ONLY = ("plaquette_check", "rotation_check")
CHAINS = ("model_check", "su_check", "u1_check")


@pytest.fixture(scope="module")
def ref_tests():
    from oracle.oracle import reference_root

    root = reference_root()
    if root is None or shutil.which("g++") is None:
        pytest.skip("reference tree or g++ not available")
    return os.path.join(root, "test")


def _build(src, out):
    cmd = ["g++", "-std=c++23", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{INC}", f"-I{os.path.join(INC, 'umc', 'compat')}",
           src, f"-L{PKG}", "-lumc_b200", f"-Wl,-rpath,{PKG}", "-o", out]
    return subprocess.run(cmd, capture_output=True, text=True)


@pytest.mark.parametrize("name", HOST_ONLY + CHAINS)
def test_reference_program_builds_and_runs(ref_tests, umc, tmp_path, name):
    out = str(tmp_path / name)
    r = _build(os.path.join(ref_tests, name + ".cpp"), out)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=600)
    if name in HOST_ONLY or umc.device_count() > 0:
        assert r.returncode == 0, r.stdout + r.stderr
        assert "ok" in r.stdout + r.stderr
    else:
        assert r.returncode != 0
        assert "no CUDA device" in r.stderr


def test_reference_host_model_is_refused_with_the_drivers_message(ref_tests, umc, tmp_path):
    r = _build(os.path.join(ref_tests, "graph_check.cpp"), str(tmp_path / "graph_check"))
    assert r.returncode != 0
    assert "runs on the device through umc/device.cuh" in r.stderr


def test_every_reference_header_has_a_compat_header(ref_tests):
    """include/umc/compat holds a header at each of the reference's include
    paths, and each one alone compiles (with the names it declares)."""
    root = os.path.dirname(ref_tests)
    compat = os.path.join(INC, "umc", "compat")
    paths = []
    for d, _, files in os.walk(root):
        if os.path.relpath(d, root).split(os.sep)[0] == "test":
            continue
        paths += [os.path.relpath(os.path.join(d, f), root) for f in files if f.endswith(".hpp")]
    assert paths
    missing = [p for p in paths if not os.path.isfile(os.path.join(compat, p))]
    assert not missing, missing
    for p in sorted(paths):
        r = subprocess.run(["g++", "-std=c++23", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", f"-I{INC}",
                            f"-I{compat}", "-x", "c++", "-"], input=f"#include <{p}>\n", capture_output=True,
                           text=True)
        assert r.returncode == 0, (p, r.stderr)
