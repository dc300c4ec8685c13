"""Generates tests/golden/golden.npz by running the REFERENCE library's own code
(its headers compiled into oracle/_ref/libumc_ref.so by oracle/Makefile).

Run from the repository root where the reference tree is mounted:

    make -C oracle ref && python tests/golden/make_golden.py

Every array is an input or an output of the reference driver on small seeded
problems; tests/test_oracle.py checks the C restatement against them, and the
GPU parity tests use the same set-ups.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from helpers import (  # noqa: E402
    checker_position,
    cubic_edges,
    link_class_position,
    random_unit_vectors,
    relabel_cells,
    relabel_edges,
    slot_edges,
    square_edges,
    square_plaquette_cells,
)
from oracle.oracle import TAG_SITE, Reference  # noqa: E402


def main():
    r = Reference()
    g = {}

    # ---- RNG: the reference Pcg32 itself, and keyed streams built from it
    for seed, stream in [(42, 54), (1, 0), (2026, 1), (2**63 + 5, 2**40 + 3)]:
        g[f"pcg_{seed}_{stream}"] = r.pcg32_draws(seed, stream, 64)
    keys = np.array([[1, 0, TAG_SITE(0), 0], [1, 7, TAG_SITE(0), 4095], [99, 123456789, 1, 2**31 + 7],
                     [2**60, 2**40, 2, 0], [5, 3, TAG_SITE(9), 1234]], np.uint64)
    g["key_list"] = keys
    g["key_draws"] = np.stack([r.key_draws(int(a), int(b), int(c), int(d), 16) for a, b, c, d in keys])

    # ---- tables
    for Lx, Ly in [(1, 1), (1, 4), (2, 2), (4, 4), (3, 5)]:
        st, off, bonds = r.square_lattice(Lx, Ly)
        assert st == 0
        g[f"square_{Lx}x{Ly}_off"] = off
        g[f"square_{Lx}x{Ly}_bonds"] = bonds
    st, cells, off, ic, iw = r.hypercubic(2)
    assert st == 0
    g["hyper2_cells"], g["hyper2_off"], g["hyper2_inc_cell"], g["hyper2_inc_which"] = cells, off, ic, iw

    # ---- Ising 8x8, colour-major relabelled, beta 0.44, cold start
    L = 8
    ei, ej = relabel_edges(*square_edges(L, L), checker_position(L, L))
    g["ising8_ei"], g["ising8_ej"] = ei, ej
    s0 = np.ones(L * L, np.int8)
    s, E, M = r.ising_metropolis(L * L, ei, ej, 1, 0.44, 1, 0, 50, s0)
    g["ising8_metro_spins"], g["ising8_metro_E"], g["ising8_metro_M"] = s, E, M
    s, sizes, E, M = r.ising_wolff(L * L, ei, ej, 1, 0.44, 3, 0, 100, s0)
    g["ising8_wolff_spins"], g["ising8_wolff_sizes"], g["ising8_wolff_E"], g["ising8_wolff_M"] = s, sizes, E, M
    # antiferromagnet J=-1 from a random start
    s0r = np.where(np.random.default_rng(3).random(L * L) < 0.5, -1, 1).astype(np.int8)
    g["ising8_s0r"] = s0r
    s, E, M = r.ising_metropolis(L * L, ei, ej, -1, 0.7, 11, 5, 20, s0r)
    g["ising8_afm_spins"], g["ising8_afm_E"], g["ising8_afm_M"] = s, E, M

    # ---- weighted Ising (test/graph_check.cpp's IsingGraph on PairGraph<double>):
    # 40 sites, 100 random edges (duplicates kept), couplings +-1 times a weight,
    # random start; the Wolff bond in slot a keyed by its edge index
    rng = np.random.default_rng(31)
    e = rng.integers(0, 40, (120, 2))
    e = e[e[:, 0] != e[:, 1]][:100].astype(np.uint32)
    c = rng.choice([-1.0, 1.0], len(e)) * rng.uniform(0.5, 1.5, len(e))
    g["wising_ei"], g["wising_ej"], g["wising_c"] = e[:, 0].copy(), e[:, 1].copy(), c
    s0 = np.where(rng.random(40) < 0.5, -1.0, 1.0)
    g["wising_s0"] = s0
    s, E = r.weighted_ising_metropolis(40, e[:, 0], e[:, 1], c, 0.6, 13, 0, 20, s0)
    g["wising_metro_s"], g["wising_metro_E"] = s, E
    st, off, bonds = r.pair_graph(40, e[:, 0], e[:, 1])
    slot = slot_edges(off, e[:, 0], e[:, 1])
    s, sizes, E = r.weighted_ising_wolff(40, e[:, 0], e[:, 1], c, slot, 0.6, 14, 0, 50, s0)
    g["wising_wolff_s"], g["wising_wolff_sizes"], g["wising_wolff_E"] = s, sizes, E

    # ---- VectorSpin<3> on a 4^3 cubic lattice
    L = 4
    n = L**3
    ei, ej = relabel_edges(*cubic_edges(L, L, L), checker_position(L, L, L))
    g["o3_ei"], g["o3_ej"] = ei, ej
    v0 = random_unit_vectors(n, 3, 7)
    g["o3_v0"] = v0
    for name, prop, delta in [("sphere", 0, 0.0), ("rot", 1, 0.5)]:
        v, obs = r.vector_metropolis(3, n, ei, ej, 1.0, 0.693, prop, delta, 5, 0, 3, v0)
        g[f"o3_metro_{name}_v"], g[f"o3_metro_{name}_obs"] = v, obs
    v, sizes, obs = r.vector_wolff(3, n, ei, ej, 1.0, 0.693, 9, 0, 20, v0)
    g["o3_wolff_v"], g["o3_wolff_sizes"], g["o3_wolff_obs"] = v, sizes, obs

    # ---- XY: VectorSpin<2> with LocalRotation, and the angle model with U1Shift
    L = 8
    ei, ej = relabel_edges(*square_edges(L, L), checker_position(L, L))
    g["xy8_ei"], g["xy8_ej"] = ei, ej
    v0 = random_unit_vectors(L * L, 2, 11)
    g["xy8_v0"] = v0
    v, obs = r.vector_metropolis(2, L * L, ei, ej, 1.0, 1.1, 1, 1.0, 4, 0, 4, v0)
    g["xy8_rot_v"], g["xy8_rot_obs"] = v, obs
    th0 = np.random.default_rng(12).uniform(0, 2 * np.pi, L * L)
    g["xy8_th0"] = th0
    th, obs = r.xy_metropolis(L * L, ei, ej, 1.0, 1.1, 1.0, 4, 0, 4, th0)
    g["xy8_angle_th"], g["xy8_angle_obs"] = th, obs

    # ---- U(1): 2D L=4 (hits 2) and 4D L=2, links relabelled by (mu, parity)
    L = 4
    cells = relabel_cells(square_plaquette_cells(L), link_class_position(L, 2))
    g["u1_2d_cells"] = cells
    th0 = np.random.default_rng(21).uniform(-np.pi, np.pi, 2 * L * L)
    g["u1_2d_th0"] = th0
    th, obs = r.u1_metropolis(cells, 2.0, 1.0, 0.5, 2, 6, 0, 3, th0)
    g["u1_2d_th"], g["u1_2d_obs"] = th, obs
    L = 2
    st, hcells, *_ = r.hypercubic(L)
    cells = relabel_cells(hcells, link_class_position(L, 4))
    g["u1_4d_cells"] = cells
    th0 = np.random.default_rng(22).uniform(-np.pi, np.pi, 4 * L**4)
    g["u1_4d_th0"] = th0
    th, obs = r.u1_metropolis(cells, 1.3, 1.0, 0.7, 1, 8, 0, 2, th0)
    g["u1_4d_th"], g["u1_4d_obs"] = th, obs

    # ---- SU(N) on the 4D L=2 complex: random links from the reference's SUShift
    for N in (2, 3):
        nl = 4 * L**4
        eye = np.eye(N, dtype=np.complex128)
        links = np.stack([r.su_shift(N, 1.5, 31 + N, 0, 3, i, eye) for i in range(nl)])
        g[f"su{N}_u0"] = links
        out, obs = r.su_metropolis(N, cells, 2.0, 1.0, 0.3, 2, 40 + N, 0, 1, links)
        g[f"su{N}_u"], g[f"su{N}_obs"] = out, obs
        a = np.random.default_rng(50 + N).normal(size=(N, N)) + 1j * np.random.default_rng(60 + N).normal(size=(N, N))
        a = 0.9 * (a - a.conj().T)  # anti-Hermitian with norm > 0.5 (squarings exercised)
        g[f"su{N}_expm_in"], g[f"su{N}_expm_out"] = a, r.su_expm(N, a)

    out = os.path.join(ROOT, "tests", "golden", "golden.npz")
    np.savez_compressed(out, **g)
    print(f"wrote {out}: {len(g)} arrays, {os.path.getsize(out)} bytes")


if __name__ == "__main__":
    main()
