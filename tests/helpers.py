"""Shared set-up for the parity tests: lattices, colour-major relabelling and
seeded states, computed independently of the engine (numpy only)."""
from __future__ import annotations

import numpy as np


def square_edges(Lx: int, Ly: int):
    """square_lattice's edge list (lattice/square.hpp:27-35)."""
    ei, ej = [], []
    for y in range(Ly):
        for x in range(Lx):
            i = y * Lx + x
            if Lx > 1:
                ei.append(i)
                ej.append(y * Lx + (x + 1) % Lx)
            if Ly > 1:
                ei.append(i)
                ej.append(((y + 1) % Ly) * Lx + x)
    return np.array(ei, np.uint32), np.array(ej, np.uint32)


def cubic_edges(Lx: int, Ly: int, Lz: int):
    ei, ej = [], []
    for z in range(Lz):
        for y in range(Ly):
            for x in range(Lx):
                i = (z * Ly + y) * Lx + x
                if Lx > 1:
                    ei.append(i)
                    ej.append((z * Ly + y) * Lx + (x + 1) % Lx)
                if Ly > 1:
                    ei.append(i)
                    ej.append((z * Ly + (y + 1) % Ly) * Lx + x)
                if Lz > 1:
                    ei.append(i)
                    ej.append((((z + 1) % Lz) * Ly + y) * Lx + x)
    return np.array(ei, np.uint32), np.array(ej, np.uint32)


def checker_position(Lx: int, Ly: int, Lz: int = 1):
    """Colour-major index of every site of an even periodic lattice:
    colour (x+y+z)&1 first, then site/2."""
    n = Lx * Ly * Lz
    s = np.arange(n)
    x, y, z = s % Lx, (s // Lx) % Ly, s // (Lx * Ly)
    c = (x + y + z) & 1
    return (c * (n // 2) + s // 2).astype(np.uint32)


def link_class_position(L: int, dim: int):
    """Colour-major index of every link of an even periodic plaquette complex
    (links mu*L^dim + site): class 2*mu + parity, then site/2."""
    V = L ** dim
    i = np.arange(dim * V)
    mu, s = i // V, i % V
    par = np.zeros_like(s)
    r = s.copy()
    for _ in range(dim):
        par += r % L
        r //= L
    cls = 2 * mu + (par & 1)
    return (cls * (V // 2) + s // 2).astype(np.uint32)


def relabel_edges(ei, ej, position):
    return position[ei].astype(np.uint32), position[ej].astype(np.uint32)


def relabel_cells(cells, position):
    return position[np.asarray(cells)].astype(np.uint32)


def to_colour_major(values, position):
    """values[site] -> out[position[site]]."""
    out = np.empty_like(values)
    out[position] = values
    return out


def from_colour_major(values, position):
    return values[position]


def random_unit_vectors(n: int, N: int, seed: int):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, N))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


def square_plaquette_cells(L: int):
    L2 = L * L
    cells = []
    for y in range(L):
        for x in range(L):
            cells.append([y * L + x, L2 + y * L + (x + 1) % L, ((y + 1) % L) * L + x, L2 + y * L + x])
    return np.array(cells, np.uint32)


def mlp_init(seed: int, scale: float = 1.0):
    """Random parameters of the 3-64-64-16 proposal network (He-style scale),
    packed W1[3][64], b1, W2[64][64], b2, W3[64][16], b3."""
    rng = np.random.default_rng(seed)
    W1 = rng.standard_normal((3, 64)) * np.sqrt(2 / 3) * scale
    b1 = rng.standard_normal(64) * 0.1
    W2 = rng.standard_normal((64, 64)) * np.sqrt(2 / 64) * scale
    b2 = rng.standard_normal(64) * 0.1
    W3 = rng.standard_normal((64, 16)) * np.sqrt(1 / 64) * scale
    b3 = rng.standard_normal(16) * 0.1
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3.ravel(), b3]).astype(np.float32).astype(np.float64)


def device_csr(g):
    """The CSR of PairTables: row k holds the bonds of the site at colour-major
    position k, as positions; and for every slot the key of its bond (the slot
    of the bond in the row of its lower endpoint)."""
    off, bonds = g.csr()
    _, _, pos = g.colouring()
    order = np.argsort(pos)
    deg = np.diff(off)[order]
    doff = np.concatenate([[0], np.cumsum(deg)]).astype(np.uint32)
    dbonds = np.concatenate([pos[bonds[off[i]:off[i + 1]]] for i in order]).astype(np.uint32)
    rows = np.repeat(np.arange(len(order)), deg)
    key = np.arange(len(dbonds), dtype=np.uint32)
    for a in np.nonzero(rows > dbonds)[0]:
        i, j = rows[a], dbonds[a]
        # a duplicated bond: the m-th copy in i's row pairs with the m-th in j's
        m = int(np.count_nonzero(dbonds[doff[i]:a] == j))
        back = doff[j] + np.nonzero(dbonds[doff[j]:doff[j + 1]] == i)[0]
        key[a] = back[m]
    return pos, doff, dbonds, key


def slot_edges(off, ei, ej, symmetric=True):
    """The input edge of every CSR slot, replaying PairGraph's scatter
    (lattice/pair_graph.hpp:77-81): rows filled in edge order."""
    pos = np.array(off[:-1], np.int64)
    slot = np.zeros(int(off[-1]), np.uint32)
    for e, (i, j) in enumerate(zip(ei, ej)):
        slot[pos[i]] = e
        pos[i] += 1
        if symmetric:
            slot[pos[j]] = e
            pos[j] += 1
    return slot
