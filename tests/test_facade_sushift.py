"""The facade's SU(N) link proposal on the host (include/umc/dof.hpp,
SUShift<N>::sample, the expm of sun_detail) against the reference's own
SUShift<N> (include/UniversalMC/dof.hpp of the reference, compiled in the
reference harness), on the same keyed streams: the facade program in
tests/cpp/facade_sushift_check.cpp reads the keys and current links, the
reference harness proposes from the same ones."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "universal_classical_montecarlo_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "facade_sushift_check.cpp")


@pytest.fixture(scope="module")
def sushift_binary(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("sushift") / "facade_sushift_check")
    cmd = [cxx, "-std=c++23", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{os.path.join(ROOT, 'include')}", SRC,
           f"-L{PKG}", "-lumc_b200", f"-Wl,-rpath,{PKG}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def _random_su(rng, n):
    """A random SU(n) matrix: QR of a complex Gaussian, phases fixed, det 1."""
    z = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    q, r = np.linalg.qr(z)
    q = q * (np.diag(r) / np.abs(np.diag(r)))
    return q / np.linalg.det(q) ** (1.0 / n)


@pytest.mark.parametrize("n", [2, 3])
def test_facade_sushift_matches_reference(sushift_binary, ref, n):
    rng = np.random.default_rng(20 + n)
    cases = []
    for k in range(64):
        width = [0.05, 0.3, 1.0, 2.5][k % 4]
        seed, counter = int(rng.integers(1, 2**63)), int(rng.integers(0, 2**40))
        tag, id_ = int(rng.integers(0, 2**32)), int(rng.integers(0, 2**32))
        cur = np.eye(n, dtype=np.complex128) if k < 4 else _random_su(rng, n)
        cases.append((width, seed, counter, tag, id_, cur))
    lines = []
    for width, seed, counter, tag, id_, cur in cases:
        lines.append(f"{n} {width!r} {seed} {counter} {tag} {id_}")
        lines += [f"{float(v.real)!r} {float(v.imag)!r}" for v in cur.reshape(-1)]
    r = subprocess.run([sushift_binary], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout.split("\n")
    assert out[len(cases) * n * n].startswith("unitarity")
    assert float(out[len(cases) * n * n].split()[1]) < 1e-12
    vals = np.array([[float(x) for x in line.split()] for line in out[: len(cases) * n * n]])
    got = (vals[:, 0] + 1j * vals[:, 1]).reshape(len(cases), n, n)
    worst = 0.0
    for k, (width, seed, counter, tag, id_, cur) in enumerate(cases):
        want = ref.su_shift(n, width, seed, counter, tag, id_, cur)
        worst = max(worst, float(np.max(np.abs(got[k] - want))))
        # a proposal moves the link: the same stream gives the same move
        assert not np.allclose(want, cur)
    # the same uniforms, the same generator matrix and the same series in the
    # same order: bit-identical on the host
    assert worst == 0.0, worst
