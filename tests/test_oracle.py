"""The CPU oracle (oracle/umc_oracle.c) against the reference's own outputs.

Golden vectors come from tests/golden/make_golden.py, which runs the reference
headers (rng.hpp, driver.hpp, example/, model/, term/) compiled into
oracle/_ref.  Where that library is present the same comparisons also run live
on fresh seeds.  Known-answer checks restate the reference's tests
(test/model_check.cpp, test/graph_check.cpp, test/su_check.cpp,
test/u1_check.cpp) with the oracle.
"""
import math

import numpy as np
import pytest

from helpers import (checker_position, cubic_edges, link_class_position, random_unit_vectors,
                     relabel_cells, relabel_edges, square_edges, square_plaquette_cells)
from oracle.oracle import TAG_SITE


# ------------------------------------------------------------------------ RNG
def test_pcg32_matches_reference_vectors(oracle, golden):
    for key in golden:
        if key.startswith("pcg_"):
            _, seed, stream = key.split("_")
            np.testing.assert_array_equal(oracle.pcg32_draws(int(seed), int(stream), 64), golden[key])


def test_pcg32_known_answer(oracle):
    # rng.hpp:14-40 is PCG-XSH-RR with the standard seeding recipe; its demo
    # stream (seed 42, stream 54) starts 0xa15c02b7 0x7b47f409 0xba1d3330.
    np.testing.assert_array_equal(oracle.pcg32_draws(42, 54, 3), [0xA15C02B7, 0x7B47F409, 0xBA1D3330])


def test_keyed_streams_match_reference(oracle, golden):
    for (s, c, t, i), want in zip(golden["key_list"], golden["key_draws"]):
        np.testing.assert_array_equal(oracle.key_draws(int(s), int(c), int(t), int(i), 16), want)


def test_keyed_stream_is_reference_pcg32(oracle):
    # a keyed stream is exactly Pcg32(id_seed(key_seed, id), 0) of rng.hpp
    for s, c, t, i in [(1, 0, TAG_SITE(0), 5), (77, 9, 2, 0), (3, 2**40, 1, 2**32 - 1)]:
        ks = oracle.key_seed(s, c, t)
        np.testing.assert_array_equal(oracle.key_draws(s, c, t, i, 8), oracle.pcg32_draws(oracle.id_seed(ks, i), 0, 8))


def test_stream_id_is_a_bijection_on_a_sample(oracle):
    ids = np.arange(0, 1 << 16)
    h = np.array([oracle.stream_id(int(i)) for i in ids])
    assert len(np.unique(h)) == len(ids)


# --------------------------------------------------------------------- tables
@pytest.mark.parametrize("Lx,Ly", [(1, 1), (1, 4), (2, 2), (4, 4), (3, 5)])
def test_square_lattice_csr_matches_reference(oracle, golden, Lx, Ly):
    st, ei, ej = oracle.square_edges(Lx, Ly)
    assert st == 0
    st, off, bonds, _ = oracle.pair_graph(Lx * Ly, ei, ej)
    assert st == 0
    np.testing.assert_array_equal(off, golden[f"square_{Lx}x{Ly}_off"])
    np.testing.assert_array_equal(bonds, golden[f"square_{Lx}x{Ly}_bonds"])


def test_square_lattice_degrees(oracle):
    # test/model_check.cpp:83-94
    for Lx, Ly, deg in [(1, 1, 0), (1, 4, 2), (2, 2, 4), (4, 4, 4)]:
        _, ei, ej = oracle.square_edges(Lx, Ly)
        _, off, _, _ = oracle.pair_graph(Lx * Ly, ei, ej)
        assert (np.diff(off) == deg).all()


def test_pair_graph_errors(oracle):
    # test/graph_check.cpp:194-214 and lattice/pair_graph.hpp:49-60
    st, off, _, _ = oracle.pair_graph(2, [0, 0], [1, 1])
    assert st == 0 and list(np.diff(off)) == [2, 2]  # duplicates kept
    st, off, b, _ = oracle.pair_graph(3, [], [])
    assert st == 0 and (off == 0).all()
    st, off, _, _ = oracle.pair_graph(2, [0], [1], symmetric=False)
    assert list(np.diff(off)) == [1, 0]
    assert oracle.pair_graph(2, [0], [0])[0] == -2  # self-loop: invalid_argument
    assert oracle.pair_graph(2, [0], [2])[0] == -1  # out_of_range


def test_hypercubic_matches_reference(oracle, golden):
    cells = oracle.hypercubic_cells(2)
    np.testing.assert_array_equal(cells, golden["hyper2_cells"])
    st, off, ic, iw = oracle.cell_incidence(4 * 16, cells)
    np.testing.assert_array_equal(off, golden["hyper2_off"])
    np.testing.assert_array_equal(ic, golden["hyper2_inc_cell"])
    np.testing.assert_array_equal(iw, golden["hyper2_inc_which"])


def test_live_tables_match_reference(oracle, ref):
    rng = np.random.default_rng(0)
    n, m = 50, 140
    ei = rng.integers(0, n, m).astype(np.uint32)
    ej = (ei + rng.integers(1, n, m)).astype(np.uint32) % n
    for sym in (True, False):
        st, off, bonds, _ = oracle.pair_graph(n, ei, ej, sym)
        st2, off2, bonds2 = ref.pair_graph(n, ei, ej, sym)
        assert st == st2 == 0
        np.testing.assert_array_equal(off, off2)
        np.testing.assert_array_equal(bonds, bonds2)
    cells = oracle.hypercubic_cells(3)
    st, off, ic, iw = oracle.cell_incidence(4 * 81, cells)
    st2, cells2, off2, ic2, iw2 = ref.hypercubic(3)
    np.testing.assert_array_equal(cells, cells2)
    np.testing.assert_array_equal(off, off2)
    np.testing.assert_array_equal(ic, ic2)
    np.testing.assert_array_equal(iw, iw2)


def test_closed_form_colourings_are_valid(oracle):
    for dims in [(8, 8, 1), (4, 4, 4), (2, 2, 1), (2, 6, 1)]:
        ei, ej = cubic_edges(*dims)
        n = int(np.prod(dims))
        _, off, bonds, _ = oracle.pair_graph(n, ei, ej)
        pos = checker_position(*dims)
        assert oracle.check_colouring(off, bonds, (pos >= n // 2).astype(np.uint32))
    for L, dim in [(2, 4), (4, 4), (4, 2), (6, 2)]:
        cells = oracle.hypercubic_cells(L) if dim == 4 else oracle.square_plaquette_cells(L)
        pos = link_class_position(L, dim)
        cls = pos // (L**dim // 2)
        assert oracle.check_cell_colouring(dim * L**dim, cells, cls)


# ---------------------------------------------------------------------- Ising
def _csr(oracle, n, ei, ej):
    st, off, bonds, slot = oracle.pair_graph(n, ei, ej)
    assert st == 0
    return off, bonds, slot


def test_ising_metropolis_golden(oracle, golden):
    off, bonds, _ = _csr(oracle, 64, golden["ising8_ei"], golden["ising8_ej"])
    s, E, M = oracle.ising_metropolis(off, bonds, 1, 0.44, 1, 0, 50, np.ones(64, np.int8))
    np.testing.assert_array_equal(s, golden["ising8_metro_spins"])
    np.testing.assert_array_equal(E, golden["ising8_metro_E"])
    np.testing.assert_array_equal(M, golden["ising8_metro_M"])
    s, E, M = oracle.ising_metropolis(off, bonds, -1, 0.7, 11, 5, 20, golden["ising8_s0r"])
    np.testing.assert_array_equal(s, golden["ising8_afm_spins"])
    np.testing.assert_array_equal(E, golden["ising8_afm_E"])


def test_ising_wolff_golden(oracle, golden):
    off, bonds, slot = _csr(oracle, 64, golden["ising8_ei"], golden["ising8_ej"])
    s, sizes, E, M = oracle.ising_wolff(off, bonds, slot, 1, 0.44, 3, 0, 100, np.ones(64, np.int8))
    np.testing.assert_array_equal(s, golden["ising8_wolff_spins"])
    np.testing.assert_array_equal(sizes, golden["ising8_wolff_sizes"])
    np.testing.assert_array_equal(E, golden["ising8_wolff_E"])
    np.testing.assert_array_equal(M, golden["ising8_wolff_M"])


def test_ising_live_against_reference(oracle, ref):
    for (Lx, Ly), beta, J in [((6, 10), 0.35, 1), ((3, 5), 0.5, 2), ((2, 2), 0.2, 1)]:
        n = Lx * Ly
        ei, ej = square_edges(Lx, Ly)
        perm = np.random.default_rng(n).permutation(n).astype(np.uint32)  # any relabelling
        ei, ej = relabel_edges(ei, ej, perm)
        off, bonds, slot = _csr(oracle, n, ei, ej)
        s0 = np.where(np.random.default_rng(1).random(n) < 0.5, -1, 1).astype(np.int8)
        a = oracle.ising_metropolis(off, bonds, J, beta, 77, 3, 40, s0)
        b = ref.ising_metropolis(n, ei, ej, J, beta, 77, 3, 40, s0)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
        a = oracle.ising_wolff(off, bonds, slot, J, beta, 5, 0, 60, s0)
        b = ref.ising_wolff(n, ei, ej, J, beta, 5, 0, 60, s0)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_ising_exact_4x4_known_answer(oracle):
    # test/model_check.cpp:171-196: exact E/site at beta=0.3 on 4x4 is -0.8440540736
    ei, ej = square_edges(4, 4)
    off, bonds, slot = _csr(oracle, 16, ei, ej)
    s, _, _ = oracle.ising_metropolis(off, bonds, 1, 0.3, 11, 0, 2000, np.ones(16, np.int8))
    _, E, _ = oracle.ising_metropolis(off, bonds, 1, 0.3, 11, 2000, 4000, s)
    assert abs(E.mean() / 16 - (-0.8440540736)) < 0.03
    s, _, _, _ = oracle.ising_wolff(off, bonds, slot, 1, 0.3, 12, 0, 2000, np.ones(16, np.int8))
    _, _, E, _ = oracle.ising_wolff(off, bonds, slot, 1, 0.3, 12, 2000, 20000, s)
    assert abs(E.mean() / 16 - (-0.8440540736)) < 0.05


def test_ising_onsager_16x16_known_answer(oracle):
    # test/graph_check.cpp:153-192 (Onsager infinite-volume energy at beta=0.3)
    beta = 0.3
    tb = math.tanh(2 * beta)
    u = -(1 / math.tanh(2 * beta)) * (1 + (2 / math.pi) * (2 * tb * tb - 1) * 2.307624577366968)
    ei, ej = relabel_edges(*square_edges(16, 16), checker_position(16, 16))
    off, bonds, slot = _csr(oracle, 256, ei, ej)
    s, _, _ = oracle.ising_metropolis(off, bonds, 1, beta, 2026, 0, 300, np.ones(256, np.int8))
    s, Em, _ = oracle.ising_metropolis(off, bonds, 1, beta, 2026, 300, 2000, s)
    e_mc = Em.mean() / 256
    s, _, Ew, _ = oracle.ising_wolff(off, bonds, slot, 1, beta, 2027, 0, 20000, s)
    e_w = Ew[200:].mean() / 256
    assert abs(e_mc - u) < 0.03 and abs(e_w - u) < 0.03 and abs(e_mc - e_w) < 0.04


# ----------------------------------------------------------------- VectorSpin
def test_vector_golden(oracle, golden):
    off, bonds, slot = _csr(oracle, 64, golden["o3_ei"], golden["o3_ej"])
    for name, prop, delta in [("sphere", 0, 0.0), ("rot", 1, 0.5)]:
        v, obs, _ = oracle.vector_metropolis(3, off, bonds, 1.0, 0.693, prop, delta, 5, 0, 3, golden["o3_v0"])
        np.testing.assert_array_equal(v, golden[f"o3_metro_{name}_v"])
        np.testing.assert_array_equal(obs, golden[f"o3_metro_{name}_obs"])
    v, sizes, obs, _ = oracle.vector_wolff(3, off, bonds, slot, 1.0, 0.693, 9, 0, 20, golden["o3_v0"])
    np.testing.assert_array_equal(v, golden["o3_wolff_v"])
    np.testing.assert_array_equal(sizes, golden["o3_wolff_sizes"])
    np.testing.assert_array_equal(obs, golden["o3_wolff_obs"])
    off, bonds, _ = _csr(oracle, 64, golden["xy8_ei"], golden["xy8_ej"])
    v, obs, _ = oracle.vector_metropolis(2, off, bonds, 1.0, 1.1, 1, 1.0, 4, 0, 4, golden["xy8_v0"])
    np.testing.assert_array_equal(v, golden["xy8_rot_v"])
    th, obs, _ = oracle.xy_metropolis(off, bonds, 1.0, 1.1, 1.0, 4, 0, 4, golden["xy8_th0"])
    np.testing.assert_array_equal(th, golden["xy8_angle_th"])
    np.testing.assert_array_equal(obs, golden["xy8_angle_obs"])


@pytest.mark.parametrize("N", [1, 2, 3, 4])
def test_vector_live_against_reference(oracle, ref, N):
    ei, ej = relabel_edges(*square_edges(6, 6), checker_position(6, 6))
    off, bonds, slot = _csr(oracle, 36, ei, ej)
    v0 = random_unit_vectors(36, N, N)
    for prop in ([0] if N == 1 else [0, 1]):
        a, oa, _ = oracle.vector_metropolis(N, off, bonds, 0.9, 0.8, prop, 0.7, 3, 2, 5, v0)
        b, ob = ref.vector_metropolis(N, 36, ei, ej, 0.9, 0.8, prop, 0.7, 3, 2, 5, v0)
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(oa, ob)
    a, za, oa, _ = oracle.vector_wolff(N, off, bonds, slot, 0.9, 0.8, 4, 0, 30, v0)
    b, zb, ob = ref.vector_wolff(N, 36, ei, ej, 0.9, 0.8, 4, 0, 30, v0)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(za, zb)


def test_heisenberg_metropolis_vs_wolff_known_answer(oracle):
    # test/model_check.cpp:198-222: two algorithms agree within 0.05 on 4x4, beta 0.3
    ei, ej = square_edges(4, 4)
    off, bonds, slot = _csr(oracle, 16, ei, ej)
    v0 = np.tile([0.0, 0.0, 1.0], (16, 1))
    v, _, _ = oracle.vector_metropolis(3, off, bonds, 1.0, 0.3, 0, 0, 13, 0, 2000, v0)
    _, obs, _ = oracle.vector_metropolis(3, off, bonds, 1.0, 0.3, 0, 0, 13, 2000, 4000, v)
    e_m = obs[:, 0].mean() / 16
    v, _, _, _ = oracle.vector_wolff(3, off, bonds, slot, 1.0, 0.3, 14, 0, 2000, v0)
    _, _, obs, _ = oracle.vector_wolff(3, off, bonds, slot, 1.0, 0.3, 14, 2000, 20000, v)
    assert abs(obs[:, 0].mean() / 16 - e_m) < 0.05


# ---------------------------------------------------------------------- gauge
def test_u1_golden(oracle, golden):
    for tag, n, mb, w, hits, seed, sweeps in [("2d", 32, 2.0, 0.5, 2, 6, 3), ("4d", 64, 1.3, 0.7, 1, 8, 2)]:
        cells = golden[f"u1_{tag}_cells"]
        inc = oracle.cell_incidence(n, cells)[1:]
        th, obs, _ = oracle.u1_metropolis(cells, inc, mb, 1.0, w, hits, seed, 0, sweeps, golden[f"u1_{tag}_th0"])
        np.testing.assert_array_equal(th, golden[f"u1_{tag}_th"])
        np.testing.assert_array_equal(obs, golden[f"u1_{tag}_obs"])


def test_su_golden(oracle, golden):
    cells = golden["u1_4d_cells"]
    inc = oracle.cell_incidence(64, cells)[1:]
    for N in (2, 3):
        u, obs, _ = oracle.su_metropolis(N, cells, inc, 2.0, 1.0, 0.3, 2, 40 + N, 0, 1, golden[f"su{N}_u0"])
        np.testing.assert_array_equal(u, golden[f"su{N}_u"])
        np.testing.assert_array_equal(obs, golden[f"su{N}_obs"])
        np.testing.assert_array_equal(oracle.su_expm(N, golden[f"su{N}_expm_in"]), golden[f"su{N}_expm_out"])


def test_u1_finite_difference_known_answer(oracle):
    # test/u1_check.cpp:55-76 restated: the chain's action change equals the sum
    # of accepted dE (checked through one-link sweeps on a 4D L=3 lattice).
    cells = oracle.hypercubic_cells(3)
    n = 4 * 81
    inc = oracle.cell_incidence(n, cells)[1:]
    th = np.random.default_rng(4).uniform(-np.pi, np.pi, n)
    S0 = 1.3 * len(cells) * (1 - oracle.u1_mean_plaquette(cells, th))
    th1, obs, _ = oracle.u1_metropolis(cells, inc, 1.3, 1.0, 2.0, 1, 3, 0, 1, th)
    S1 = 1.3 * len(cells) * (1 - oracle.u1_mean_plaquette(cells, th1))
    assert abs(obs[0, 0] - S1) < 1e-9 and S0 != S1


def test_su_unitarity_known_answer(oracle, golden):
    # test/su_check.cpp:22-38, :96-97: SUShift keeps links unitary
    for N in (2, 3):
        for u in golden[f"su{N}_u"]:
            assert oracle.su_unitarity_error(N, u) < 1e-12


def test_u1_limits_known_answer(oracle):
    # test/u1_check.cpp:78-95 with beta placed once: beta=0 gives <P> ~ 0,
    # large beta gives <P> > 0.9 (4D, L=4 there; L=3 here to stay fast)
    cells = oracle.hypercubic_cells(3)
    n = 4 * 81
    inc = oracle.cell_incidence(n, cells)[1:]
    th = np.zeros(n)
    _, obs, _ = oracle.u1_metropolis(cells, inc, 0.0, 1.0, 0.7, 1, 10, 0, 150, th)
    assert abs(obs[50:, 1].mean()) < 0.05
    _, obs, _ = oracle.u1_metropolis(cells, inc, 10.0, 1.0, 0.7, 1, 20, 0, 100, th)
    assert obs[50:, 1].mean() > 0.9


def test_u1_2d_live_against_reference(oracle, ref):
    L = 6
    cells = relabel_cells(square_plaquette_cells(L), link_class_position(L, 2))
    inc = oracle.cell_incidence(2 * L * L, cells)[1:]
    th0 = np.random.default_rng(5).uniform(-np.pi, np.pi, 2 * L * L)
    a, oa, _ = oracle.u1_metropolis(cells, inc, 3.0, 1.0, 0.5, 3, 9, 4, 5, th0)
    b, ob = ref.u1_metropolis(cells, 3.0, 1.0, 0.5, 3, 9, 4, 5, th0)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(oa, ob)


# --------------------------------------------- weighted Ising (bond payloads)
def _wising_setup(golden):
    ei, ej, c = golden["wising_ei"], golden["wising_ej"], golden["wising_c"]
    return ei, ej, c


def _slot_couplings(oracle, n, ei, ej, c):
    """CSR of PairGraph<double>(n, edges) and the coupling of every slot (the
    reference copies Edge::c into both directed entries)."""
    from helpers import slot_edges

    st, off, bonds, _ = oracle.pair_graph(n, ei, ej)
    assert st == 0
    slot = slot_edges(off, ei, ej)
    return off, bonds, slot, c[slot]


def test_weighted_ising_matches_reference_vectors(oracle, golden):
    """test/graph_check.cpp's IsingGraph (PairGraph<double> couplings, random
    +-J times a weight, duplicate edges) under Metropolis and Wolff."""
    ei, ej, c = _wising_setup(golden)
    off, bonds, slot, cs = _slot_couplings(oracle, 40, ei, ej, c)
    s, E, _ = oracle.weighted_ising_metropolis(off, bonds, cs, 0.6, 13, 0, 20, golden["wising_s0"])
    np.testing.assert_array_equal(s, golden["wising_metro_s"])
    np.testing.assert_allclose(E, golden["wising_metro_E"], rtol=1e-12)
    s, sizes, E = oracle.weighted_ising_wolff(off, bonds, slot, cs, 0.6, 14, 0, 50, golden["wising_s0"])
    np.testing.assert_array_equal(sizes, golden["wising_wolff_sizes"])
    np.testing.assert_array_equal(s, golden["wising_wolff_s"])
    np.testing.assert_allclose(E, golden["wising_wolff_E"], rtol=1e-12)


@pytest.mark.parametrize("seed", [1, 2])
def test_weighted_ising_matches_reference_live(oracle, ref, seed):
    rng = np.random.default_rng(100 + seed)
    n = 64
    e = rng.integers(0, n, (200, 2))
    e = e[e[:, 0] != e[:, 1]].astype(np.uint32)
    c = rng.choice([-1.0, 1.0], len(e)) * rng.uniform(0.2, 2.0, len(e))
    off, bonds, slot, cs = _slot_couplings(oracle, n, e[:, 0], e[:, 1], c)
    s0 = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    s_r, E_r = ref.weighted_ising_metropolis(n, e[:, 0], e[:, 1], c, 0.45, seed, 3, 15, s0)
    s_o, E_o, _ = oracle.weighted_ising_metropolis(off, bonds, cs, 0.45, seed, 3, 15, s0)
    np.testing.assert_array_equal(s_o, s_r)
    np.testing.assert_allclose(E_o, E_r, rtol=1e-12)
    s_r, z_r, E_r = ref.weighted_ising_wolff(n, e[:, 0], e[:, 1], c, slot, 0.45, seed, 2, 30, s0)
    s_o, z_o, E_o = oracle.weighted_ising_wolff(off, bonds, slot, cs, 0.45, seed, 2, 30, s0)
    np.testing.assert_array_equal(z_o, z_r)
    np.testing.assert_array_equal(s_o, s_r)


def test_weighted_ising_uniform_couplings_equal_the_ising_model(oracle):
    """With every coupling 1 the weighted Wolff is the plain Ising Wolff
    (example/ising.hpp, J = 1) on the same keys."""
    L = 8
    ei, ej = square_edges(L, L)
    st, off, bonds, slot = oracle.pair_graph(L * L, ei, ej)
    s0 = np.where(np.random.default_rng(4).random(L * L) < 0.5, -1, 1).astype(np.int8)
    s_i, z_i, E_i, _ = oracle.ising_wolff(off, bonds, slot, 1, 0.44, 5, 0, 40, s0)
    s_w, z_w, E_w = oracle.weighted_ising_wolff(off, bonds, slot, np.ones(len(bonds)), 0.44, 5, 0, 40,
                                                s0.astype(np.float64))
    np.testing.assert_array_equal(z_w, z_i)
    np.testing.assert_array_equal(s_w, s_i.astype(np.float64))
    np.testing.assert_array_equal(E_w, E_i)
