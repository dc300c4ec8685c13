"""The learned-proposal oracle: Bessel functions, BF16 rounding, the network and
its gradient (against torch autograd in FP64 and finite differences), the
Best-Fisher sampler (KS test against the von Mises law), and the learned
Metropolis-Hastings update against the reference Metropolis driver with the
same proposal plugged in as a user Proposal."""
import math

import numpy as np
import pytest
import scipy.special as sp
import scipy.stats as st
import torch

from helpers import link_class_position, relabel_cells, square_plaquette_cells, mlp_init

P_SIZE = 5456


def test_bessel_series_matches_scipy(oracle):
    for x in [1e-4, 0.01, 0.3, 1.0, 5.0, 20.0, 55.0, 79.9]:
        assert oracle.log_i0(x) == pytest.approx(math.log(sp.i0e(x)) + x, rel=1e-13, abs=1e-15)
        assert oracle.i1_over_i0(x) == pytest.approx(sp.i1e(x) / sp.i0e(x), rel=1e-13)


def test_bf16_rounding_matches_torch(oracle):
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.standard_normal(2000) * 10 ** rng.uniform(-6, 4, 2000), [0.0, -0.0, 1.0]])
    ref = torch.tensor(v, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    got = np.array([oracle.bf16(x) for x in v])
    np.testing.assert_array_equal(got, ref)


def _split(P):
    P = torch.as_tensor(P, dtype=torch.float64)
    return (P[0:192].view(3, 64), P[192:256], P[256:4352].view(64, 64), P[4352:4416],
            P[4416:5440].view(64, 16), P[5440:5456])


def _torch_forward(P, x, bf16=False):
    W1, b1, W2, b2, W3, b3 = _split(P)
    x = torch.as_tensor(x, dtype=torch.float64)
    r = (lambda t: t.to(torch.float32).to(torch.bfloat16).to(torch.float64)) if bf16 else (lambda t: t)
    h1 = r(torch.relu(r(x) @ r(W1) + b1))
    h2 = r(torch.relu(h1 @ r(W2) + b2))
    return h2 @ r(W3) + b3


def _torch_loss(P, x, theta):
    o = _torch_forward(P, x)
    logits, u, v, l = o[:, 0::4], o[:, 1::4], o[:, 2::4], o[:, 3::4]
    logw = torch.log_softmax(logits, dim=1)
    mu = torch.atan2(v, u)
    kappa = torch.nn.functional.softplus(l).clamp(1e-4, 80.0)
    t = torch.as_tensor(theta, dtype=torch.float64)[:, None]
    lk = logw + kappa * torch.cos(t - mu) - torch.log(torch.special.i0(kappa)) - math.log(2 * math.pi)
    return -torch.logsumexp(lk, dim=1).mean()


def _data(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-np.pi, np.pi, n)
    r = rng.uniform(0, 2, n)
    x = np.stack([np.cos(a), np.sin(a), r], 1)
    theta = rng.uniform(-np.pi, np.pi, n)
    return x, theta


@pytest.mark.parametrize("emulate", [False, True])
def test_forward_matches_torch(oracle, emulate):
    P = mlp_init(3)
    x, _ = _data(200, 1)
    got = oracle.mlp_forward(P, x, emulate=emulate)
    ref = _torch_forward(P, x, bf16=emulate).numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_gradient_matches_torch_autograd(oracle):
    P = mlp_init(5)
    x, theta = _data(300, 2)
    loss, g = oracle.mlp_loss_grad(P, x, theta, emulate=False)
    Pt = torch.tensor(P, dtype=torch.float64, requires_grad=True)
    lt = _torch_loss(Pt, x, theta)
    lt.backward()
    assert loss == pytest.approx(lt.item(), rel=1e-12)
    np.testing.assert_allclose(g, Pt.grad.numpy(), rtol=1e-9, atol=1e-12)


def test_gradient_finite_differences(oracle):
    P = mlp_init(7)
    x, theta = _data(64, 3)
    _, g = oracle.mlp_loss_grad(P, x, theta, emulate=False)
    rng = np.random.default_rng(4)
    for idx in list(rng.choice(P_SIZE, 24, replace=False)) + [191, 255, 4351, 4415, 5439, 5455]:
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[idx] += h
        Pm[idx] -= h
        fd = (oracle.mlp_loss_grad(Pp, x, theta, False, grad=False)[0] -
              oracle.mlp_loss_grad(Pm, x, theta, False, grad=False)[0]) / (2 * h)
        assert fd == pytest.approx(g[idx], rel=1e-4, abs=1e-8), idx


def test_best_fisher_closed_form_of_r():
    """r = s + sqrt(1 + s^2), s = 1/(2 kappa) equals Best-Fisher's (1 + rho^2)/(2 rho)."""
    for k in [1e-3, 0.1, 1.0, 7.0, 80.0]:
        tau = 1 + math.sqrt(1 + 4 * k * k)
        rho = (tau - math.sqrt(2 * tau)) / (2 * k)
        s = 0.5 / k
        assert s + math.sqrt(1 + s * s) == pytest.approx((1 + rho * rho) / (2 * rho), rel=1e-6)


@pytest.mark.parametrize("kappa", [1e-3, 0.05, 1.0, 4.0, 30.0, 80.0])
def test_best_fisher_sampler_is_von_mises(oracle, kappa):
    s = np.array([oracle.vm_sample(kappa, 11, 0, 6, i) for i in range(4000)])
    assert np.all(np.abs(s) <= np.pi)
    p = st.kstest(s, st.vonmises(kappa).cdf).pvalue
    assert p > 1e-4, p


def test_mixture_density_is_normalised(oracle):
    o = np.random.default_rng(5).standard_normal(16)
    t = np.linspace(-np.pi, np.pi, 20001)
    f = np.exp([oracle.vm_mixture_logpdf(o, a) for a in t])
    assert np.trapezoid(f, t) == pytest.approx(1.0, rel=1e-6)
    w, mu, k, _ = oracle.vm_mixture(o)
    assert w.sum() == pytest.approx(1.0) and np.all(k >= 1e-4) and np.all(np.abs(mu) <= np.pi)


def _u1_tables(oracle, L):
    cells = relabel_cells(square_plaquette_cells(L), link_class_position(L, 2))
    inc = oracle.cell_incidence(2 * L * L, cells)[1:]
    return cells, inc


def test_learned_update_matches_reference_driver(oracle, ref):
    L = 4
    cells, inc = _u1_tables(oracle, L)
    P = mlp_init(9)
    th0 = np.random.default_rng(6).uniform(-np.pi, np.pi, 2 * L * L)
    a, obs, _, _, acc = oracle.u1_learned_metropolis(cells, inc, P, 2.5, 1.0, 21, 3, 4, th0)
    b, pl = ref.u1_learned_metropolis(cells, inc, P, 2.5, 1.0, 21, 3, 4, th0)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(obs[:, 1], pl, rtol=1e-14)
    assert 0 < acc.sum() < acc.size  # both outcomes exercised


def test_given_outputs_reproduce_the_sweep(oracle):
    L = 6
    cells, inc = _u1_tables(oracle, L)
    P = mlp_init(10)
    th0 = np.random.default_rng(7).uniform(-np.pi, np.pi, 2 * L * L)
    a, _, ma, dump, acc = oracle.u1_learned_metropolis(cells, inc, P, 1.7, 1.0, 5, 0, 1, th0)
    b, _, mb, _, acc2 = oracle.u1_learned_metropolis(cells, inc, P, 1.7, 1.0, 5, 0, 1, th0, given_out=dump)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(acc, acc2)


def torus_plaquette(beta, n_plaq):
    """Exact <cos theta_p> of 2D U(1) on a periodic torus with n_plaq plaquettes:
    Z = sum_n I_n(beta)^n_plaq, <P> = sum_n I_n^(n_plaq-1) I_n' / sum_n I_n^n_plaq."""
    ns = np.arange(-40, 41)
    i = sp.ive(ns, beta)  # common factor e^-beta cancels
    di = 0.5 * (sp.ive(ns - 1, beta) + sp.ive(ns + 1, beta))
    return float(np.sum(i ** (n_plaq - 1) * di) / np.sum(i ** n_plaq))


def test_learned_chain_samples_the_exact_distribution(oracle, umc):
    """Any network gives a valid MH proposal: the chain's mean plaquette equals the
    exact finite-torus value (4x4, beta 1.5) within four standard errors."""
    L, beta = 4, 1.5
    cells, inc = _u1_tables(oracle, L)
    P = mlp_init(12)
    th = np.zeros(2 * L * L)
    th, _, _, _, _ = oracle.u1_learned_metropolis(cells, inc, P, beta, 1.0, 1, 0, 200, th)
    _, obs, _, _, _ = oracle.u1_learned_metropolis(cells, inc, P, beta, 1.0, 1, 200, 6000, th)
    pl = obs[:, 1]
    m, err = umc.binning_error(pl, 200)
    exact = torus_plaquette(beta, L * L)
    assert abs(m - exact) < 4 * err + 1e-3, (m, err, exact)


def test_adam_step(oracle):
    rng = np.random.default_rng(8)
    p, g = rng.standard_normal(50), rng.standard_normal(50)
    m, v = np.zeros(50), np.zeros(50)
    p1, m1, v1 = oracle.adam_step(p, g, m, v, 1, 1e-3)
    # first step of Adam moves every parameter by lr * sign(g) (up to eps)
    np.testing.assert_allclose(p1 - p, -1e-3 * np.sign(g), rtol=1e-6)
    tp = torch.tensor(p, requires_grad=True)
    opt = torch.optim.Adam([tp], lr=1e-3)
    for t, gg in enumerate([g, 2 * g, -g], start=1):
        tp.grad = torch.tensor(gg)
        opt.step()
        p, m, v = oracle.adam_step(p, gg, m, v, t, 1e-3)
    np.testing.assert_allclose(p, tp.detach().numpy(), rtol=1e-12, atol=1e-15)


def test_plain_keyed_chain_samples_the_exact_distribution(oracle, umc):
    """The counter-keyed random streams must not bias a sampler: plain U1Shift
    Metropolis on a 4 x 4 torus at beta = 1 reproduces the exact plaquette to
    within four standard errors (about 1.6e-3).  Giving all ids of a key one
    seed and a per-id stream increment missed it by 2.5e-3."""
    L, beta = 4, 1.0
    cells, inc = _u1_tables(oracle, L)
    th = np.zeros(2 * L * L)
    th, _, _ = oracle.u1_metropolis(cells, inc, beta, 1.0, 0.5, 1, 7, 0, 2000, th)
    _, obs, _ = oracle.u1_metropolis(cells, inc, beta, 1.0, 0.5, 1, 7, 2000, 1_500_000, th)
    m, err = umc.binning_error(obs[:, 1], 5000)
    exact = torus_plaquette(beta, L * L)
    assert abs(m - exact) < 4 * err, (m, err, exact)


def test_sector_plaquettes_recombine_to_the_torus_value():
    """bench.py's exact plaquette per topological sector: weighted by Z_Q
    the sector values give back the all-sector torus plaquette (character
    expansion), and the sectors differ as expected (|Q| > 0 costs action)."""
    import importlib.util
    import os

    spec = importlib.util.spec_from_file_location(
        "bench", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for beta, V in [(2.0, 16), (4.0, 64), (8.0, 4096)]:
        w = {}
        tab = bench.torus_plaquette_sectors(beta, V, range(-40, 41), weights=w)
        mix = sum(w[q] * tab[q] for q in tab) / sum(w.values())
        assert abs(mix - bench.torus_plaquette(beta, V)) < 1e-9, (beta, V, mix)
        assert tab[0] > tab[1] > tab[2] and abs(tab[1] - tab[-1]) < 1e-12
