"""Reference-style programs with user-written terms (tests/cpp/facade_user_terms.cu),
built with nvcc: the facade's Metropolis and Wolff run the user's terms on the
device through umc/device_facade.cuh.  The program compiles here; without a
GPU it fails loudly; on the GPU its fields equal the oracle's:
- XY angles, 5 sweeps, to 1e-9;
- Ising under Wolff, spins and cluster sizes bit for bit, flips and a sweep;
- U(1) plaquettes, 2 sweeps, to 1e-9;
- O(3) with LocalRotation, 2 sweeps, to 1e-9;
- SU(3) links with a plaquette term written against SULink and the
  reference's SUShift (expm on the device), 2 sweeps, to 1e-9.
The oracle runs on the colour-major device numbering with the same keys."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import device_csr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "universal_classical_montecarlo_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "facade_user_terms.cu")
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")


@pytest.fixture(scope="module")
def program(tmp_path_factory, umc):
    if not os.path.isfile(NVCC):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("facade_user") / "facade_user_terms")
    cmd = [NVCC, "-std=c++20", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "--expt-relaxed-constexpr",
           "-diag-suppress", "177", f"-I{os.path.join(ROOT, 'include')}", SRC, f"-L{PKG}", "-lumc_b200",
           "-Xlinker", f"-rpath,{PKG}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_user_term_program_compiles_and_fails_loudly_without_gpu(program, umc, tmp_path):
    assert os.path.isfile(program)
    if umc.device_count() > 0:
        pytest.skip("a GPU is present")
    r = subprocess.run([program, str(tmp_path / "out.bin")], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0  # a CUDA error surfaces as an exception, no CPU fallback


@pytest.mark.gpu
def test_user_term_program_matches_the_oracle(program, umc, oracle, tmp_path):
    path = tmp_path / "out.bin"
    r = subprocess.run([program, str(path)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
    raw = path.read_bytes()
    at = 0

    def take(dtype, n):
        nonlocal at
        a = np.frombuffer(raw, dtype, n, at)
        at += a.nbytes
        return a

    # XY: 3 + 2 sweeps from the start field, keys Pcg32(4, 0).key() = 4
    g = umc.square_lattice(32, 32)
    n = 32 * 32
    pos, doff, dbonds, key = device_csr(g)
    xy0, xy1 = take(np.float64, n), take(np.float64, n)
    cm = np.empty(n)
    cm[pos] = xy0
    t_o, _, margin = oracle.xy_metropolis(doff, dbonds, 1.0, 1.1, 1.0, 4, 0, 5, cm)
    d = np.abs(np.angle(np.exp(1j * (xy1 - t_o[pos]))))
    assert d.max() < 1e-9, d.max()

    # Ising: 12 Wolff flips with FixedAxis, keys 13
    g = umc.square_lattice(24, 24)
    n = 24 * 24
    pos, doff, dbonds, key = device_csr(g)
    s0, s1, sizes = take(np.int8, n), take(np.int8, n), take(np.uint64, 12)
    s2, mean_after = take(np.int8, n), take(np.float64, 1)[0]
    cm = np.empty(n, np.int8)
    cm[pos] = s0
    s_o, sz_o, _, _ = oracle.ising_wolff(doff, dbonds, key, 1, 0.44, 13, 0, 12, cm)
    np.testing.assert_array_equal(sizes, sz_o)
    np.testing.assert_array_equal(s1, s_o[pos])
    # Wolff::sweep: flips 12, 13, ... until the flipped sites reach the lattice
    all_sizes, touched, f, cur = list(sz_o), 0, 12, s_o
    while touched < n:
        cur, sz, _, _ = oracle.ising_wolff(doff, dbonds, key, 1, 0.44, 13, f, 1, cur)
        touched += int(sz[0])
        all_sizes.append(int(sz[0]))
        f += 1
    np.testing.assert_array_equal(s2, cur[pos])
    assert abs(mean_after - np.mean(all_sizes)) < 1e-9

    # U(1): 2 sweeps on the 4^4 plaquettes, keys 9
    cc = umc.hypercubic_plaquettes(4)
    n = cc.sites()
    _, _, pos = cc.colouring()
    rcells = pos[cc.table()]
    inc = oracle.cell_incidence(n, rcells)[1:]
    u0, u1 = take(np.float64, n), take(np.float64, n)
    cm = np.empty(n)
    cm[pos] = u0
    t_o, _, _ = oracle.u1_metropolis(rcells, inc, 1.3, 1.0, 0.7, 1, 9, 0, 2, cm)
    d = np.abs(np.angle(np.exp(1j * (u1 - t_o[pos]))))
    assert d.max() < 1e-9, d.max()

    # O(3) with the user's Heisenberg term and LocalRotation(0.6), 2 sweeps, keys 21
    g = umc.cubic_lattice(8, 8, 8)
    n = 512
    pos, doff, dbonds, key = device_csr(g)
    v0, v1 = take(np.float64, 3 * n).reshape(n, 3), take(np.float64, 3 * n).reshape(n, 3)
    cm = np.empty((n, 3))
    cm[pos] = v0
    v_o, _, margin = oracle.vector_metropolis(3, doff, dbonds, 1.0, 0.693, 1, 0.6, 21, 0, 2, cm)
    assert np.abs(v1 - v_o[pos]).max() < 1e-9
    assert abs(np.linalg.norm(v1, axis=1) - 1).max() < 1e-12

    # SU(3) with the user's plaquette term (SULink interface) and the
    # reference's SUShift(0.3), 2 sweeps at beta 5.7, keys 33: the oracle's
    # restatement of SUShift and expm (dof/sun.hpp) on the same links
    cc = umc.hypercubic_plaquettes(4)
    n = cc.sites()
    _, _, pos = cc.colouring()
    rcells = pos[cc.table()]
    inc = oracle.cell_incidence(n, rcells)[1:]
    s0 = take(np.float64, 18 * n).view(np.complex128).reshape(n, 3, 3)
    s1 = take(np.float64, 18 * n).view(np.complex128).reshape(n, 3, 3)
    assert at == len(raw)
    cm = np.empty((n, 3, 3), np.complex128)
    cm[pos] = s0
    l_o, _, margin = oracle.su_metropolis(3, rcells, inc, 5.7, 1.0, 0.3, 1, 33, 0, 2, cm)
    moved = np.abs(s1 - s0).max(axis=(1, 2)) > 0
    assert 0.2 < moved.mean() < 0.95  # a Metropolis chain, not a frozen or free one
    assert np.abs(s1 - l_o[pos]).max() < 1e-9
