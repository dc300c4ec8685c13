"""The two SU(3) exponentials of the SUShift proposal (exp(iX) for a traceless
Hermitian X, csrc/umc_gauge_kernels.cuh su_exp_i<3>), restated in FP64 numpy
and checked against scipy's matrix exponential:

- ||X|| <= 1: the series sum_k (iX)^k / k!, each power reduced by
  Cayley-Hamilton X^3 = c1 X + c0 I to a_k I + b_k X + d_k X^2, twelve terms;
- otherwise the closed form of Morningstar & Peardon (Phys. Rev. D 69, 054501
  (2004)) with f_j(-c0) = (-1)^j conj f_j(c0).

The reference itself sums the Taylor series with scaling and squaring
(dof/sun.hpp:118-146); all three agree to FP64 rounding here, so the device's
FP32 forms differ from the reference only by FP32 rounding."""
import math

import numpy as np
import pytest
import scipy.linalg as sla


def _random_x(rng, scale):
    a = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    x = (a + a.conj().T) / 2
    x -= np.trace(x) / 3 * np.eye(3)
    return x * (scale / np.linalg.norm(x, 2))


def _invariants(x):
    x2 = x @ x
    c1 = 0.5 * np.trace(x2).real
    c0 = np.trace(x @ x2).real / 3.0  # det X
    return x2, c0, c1


def series(x, terms=12):
    x2, c0, c1 = _invariants(x)
    a, b, d = 1.0, 0.0, 0.0
    f = np.array([1.0 + 0j, 0j, 0j])
    for k in range(1, terms + 1):
        a, b, d = c0 * d, a + c1 * d, b
        f += (1j ** k) / math.factorial(k) * np.array([a, b, d])
    return f[0] * np.eye(3) + f[1] * x + f[2] * x2


def closed_form(x):
    x2, c0, c1 = _invariants(x)
    neg = c0 < 0
    c13 = c1 / 3
    th = math.acos(min(abs(c0) / (2 * c13 * math.sqrt(c13)), 1.0))
    u = math.sqrt(c13) * math.cos(th / 3)
    w = math.sqrt(c1) * math.sin(th / 3)
    xi = math.sin(w) / w if abs(w) >= 0.05 else 1 - w * w / 6 * (1 - w * w / 20 * (1 - w * w / 42))
    e2iu, emiu = np.exp(2j * u), np.exp(-1j * u)
    h0 = (u * u - w * w) * e2iu + emiu * (8 * u * u * math.cos(w) + 2j * u * (3 * u * u + w * w) * xi)
    h1 = 2 * u * e2iu - emiu * (2 * u * math.cos(w) - 1j * (3 * u * u - w * w) * xi)
    h2 = e2iu - emiu * (math.cos(w) + 3j * u * xi)
    f = np.array([h0, h1, h2]) / (9 * u * u - w * w)
    if neg:
        f = np.array([np.conj(f[0]), -np.conj(f[1]), np.conj(f[2])])
    return f[0] * np.eye(3) + f[1] * x + f[2] * x2


@pytest.mark.parametrize("scale", [1e-6, 0.05, 0.2, 0.5, 1.0])
def test_series_matches_expm(scale):
    # truncation after twelve terms: about scale^13 / 13! (1.6e-10 at 1, far
    # below the FP32 rounding of the device form)
    tol = max(1e-13, 2.0 * scale**13 / math.factorial(13))
    rng = np.random.default_rng(int(scale * 1e6) + 1)
    for _ in range(200):
        x = _random_x(rng, scale)
        np.testing.assert_allclose(series(x), sla.expm(1j * x), rtol=0, atol=tol)


@pytest.mark.parametrize("scale", [0.3, 1.0, 2.0, 5.0, 10.0])
def test_closed_form_matches_expm(scale):
    rng = np.random.default_rng(int(scale * 100) + 7)
    for _ in range(200):
        x = _random_x(rng, scale)
        np.testing.assert_allclose(closed_form(x), sla.expm(1j * x), rtol=0, atol=1e-12)
        if rng.random() < 0.5:  # the c0 < 0 branch
            np.testing.assert_allclose(closed_form(-x), sla.expm(-1j * x), rtol=0, atol=1e-12)


def test_series_switch_point_covers_the_spectrum():
    # c1 <= 0.75 bounds every eigenvalue by sqrt(4 c1 / 3) <= 1
    rng = np.random.default_rng(5)
    for _ in range(500):
        x = _random_x(rng, rng.uniform(0.1, 3.0))
        _, _, c1 = _invariants(x)
        lam = np.abs(np.linalg.eigvalsh(x)).max()
        assert lam <= math.sqrt(4 * c1 / 3) + 1e-12
