"""User-written models on the GPU (include/umc/device.cuh).

examples/device_models/user_models.cu defines, the way a user would, an XY pair term, a
U(1) plaquette term, a table-free cubic O(3) ModelLike and two proposals, all
in FP64 with __host__ __device__ members, and drives them with
umc::gpu::device::Metropolis.  On the GPU every sweep is compared with the
oracle's reference-semantics driver on the colour-major relabelled tables
(same keyed streams): the field agrees to 1e-9 except at decisions that sat
within 1e-9 of their threshold and the sites those decisions touch, and the
energies from energy_at / cell_energy agree with the oracle's observables.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "examples", "device_models"))
sys.path.insert(0, HERE)

from helpers import (checker_position, cubic_edges, device_csr, random_unit_vectors, relabel_edges,  # noqa: E402
                     square_edges)

TOL = 1e-9
MARGIN = 1e-9
_vp, _d, _u64, _u32 = C.c_void_p, C.c_double, C.c_uint64, C.c_uint32
_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib(umc):
    import build_device_models

    path = build_device_models.build()
    L = C.CDLL(path)
    L.um_last_error.restype = C.c_char_p
    L.um_xy_pair.argtypes = [_vp, _d, _d, _d, _u64, _u64, _u32, _dp, _dp, C.POINTER(_u32)]
    L.um_u1_cells.argtypes = [_vp, _d, _d, _d, _u64, _u64, _u32, _dp, _dp]
    L.um_heisenberg_cubic.argtypes = [_u32, _u32, _u32, _d, _d, _u64, _u64, _u32, _dp, _dp]
    L.um_heisenberg_cubic8_base.argtypes = [_d, _d, _u64, _u64, _u32, _dp, _dp]
    return L


def _p(a):
    return a.ctypes.data_as(_dp)


def _call(lib, rc):
    assert rc == 0, lib.um_last_error().decode()


def xy_run(lib, g, theta, beta, width, seed, sweep0, n):
    th = np.array(theta, np.float64, copy=True)
    en = np.zeros(n)
    grid = _u32(0)
    _call(lib, lib.um_xy_pair(g._h, 1.0, beta, width, seed, sweep0, n, _p(th), _p(en), C.byref(grid)))
    return th, en, grid.value


def _neighbours(off, bonds, sites):
    out = set()
    for i in sites:
        out.update(bonds[off[i]:off[i + 1]].tolist())
    return out


def test_user_library_exports_and_fails_loudly_without_gpu(umc, lib):
    for name in ("um_xy_pair", "um_u1_cells", "um_heisenberg_cubic", "um_last_error"):
        assert hasattr(lib, name)
    if umc.device_count() > 0:
        pytest.skip("a GPU is present")
    g = umc.square_lattice(8, 8)
    th = np.zeros(64)
    en = np.zeros(1)
    rc = lib.um_xy_pair(g._h, 1.0, 1.0, 1.0, 1, 0, 1, _p(th), _p(en), None)
    assert rc != 0 and lib.um_last_error()  # a CUDA error, no CPU fallback


@pytest.mark.gpu
@pytest.mark.parametrize("L,sweeps", [(64, 3), (1024, 2)])
def test_user_xy_pair_model_per_sweep(umc, oracle, lib, L, sweeps):
    g = umc.square_lattice(L, L)
    n = L * L
    _, _, pos = g.colouring()
    off_o, bonds_o = oracle_csr(oracle, umc, g, pos)
    off_s, bonds_s = g.csr()
    th = np.random.default_rng(L).uniform(-np.pi, np.pi, n)
    for sweep in range(sweeps):
        cm = np.empty(n)
        cm[pos] = th
        t_o, obs_o, margin = oracle.xy_metropolis(off_o, bonds_o, 1.0, 1.1, 1.0, 4, sweep, 1, cm)
        th, en, grid = xy_run(lib, g, th, 1.1, 1.0, 4, sweep, 1)
        if L == 1024:
            assert grid * 256 < n // 2  # the grid-stride loop wraps within a class
        d = np.abs(np.angle(np.exp(1j * (th - t_o[pos]))))
        near = np.nonzero(np.abs(margin[pos]) < MARGIN)[0]
        bad = set(np.nonzero(d > TOL)[0].tolist())
        assert bad <= set(near.tolist()) | _neighbours(off_s, bonds_s, near), sorted(bad)[:10]
        assert abs(en[0] - obs_o[0, 0]) < 1e-9 * n


def oracle_csr(oracle, umc, g, pos):
    off, bonds = g.csr()
    ei = np.repeat(np.arange(len(off) - 1, dtype=np.uint32), np.diff(off))
    keep = ei < bonds  # every undirected bond once, in CSR order of its lower endpoint
    ri, rj = relabel_edges(ei[keep], bonds[keep], pos)
    st, o, b, _ = oracle.pair_graph(len(off) - 1, ri, rj)
    assert st == 0
    return o, b


@pytest.mark.gpu
def test_user_xy_runs_continue_exactly(umc, lib):
    """n sweeps in one launch equal the same sweeps split across launches
    (the counter keys the streams), and sample() records the energy after
    every sweep."""
    g = umc.square_lattice(128, 128)
    th0 = np.random.default_rng(2).uniform(-np.pi, np.pi, 128 * 128)
    a, ea, _ = xy_run(lib, g, th0, 0.9, 1.3, 8, 0, 5)
    b1, eb1, _ = xy_run(lib, g, th0, 0.9, 1.3, 8, 0, 2)
    b2, eb2, _ = xy_run(lib, g, b1, 0.9, 1.3, 8, 2, 3)
    np.testing.assert_array_equal(a, b2)
    np.testing.assert_array_equal(ea, np.concatenate([eb1, eb2]))


@pytest.mark.gpu
@pytest.mark.parametrize("kind,L,beta,width,sweeps", [("2d", 8, 2.0, 0.5, 4), ("4d", 4, 1.1, 0.7, 3),
                                                      ("4d", 6, 0.9, 1.0, 2)])
def test_user_u1_cell_model(umc, oracle, lib, kind, L, beta, width, sweeps):
    cc = umc.square_plaquettes(L) if kind == "2d" else umc.hypercubic_plaquettes(L)
    n = cc.sites()
    _, _, pos = cc.colouring()
    cells = cc.table()
    rcells = pos[cells]
    inc = oracle.cell_incidence(n, rcells)[1:]
    th0 = np.random.default_rng(L).uniform(-np.pi, np.pi, n)
    # all sweeps in one launch against the oracle's sweeps in link order
    th = th0.copy()
    E = _d(0.0)
    _call(lib, lib.um_u1_cells(cc._h, beta, 1.0, width, 3, 0, sweeps, _p(th), C.byref(E)))
    cm = np.empty(n)
    cm[pos] = th0
    t_o, obs_o, margin = oracle.u1_metropolis(rcells, inc, beta, 1.0, width, 1, 3, 0, sweeps, cm)
    d = np.abs(np.angle(np.exp(1j * (th - t_o[pos]))))
    assert d.max() < TOL, d.max()
    assert abs(E.value - obs_o[-1, 0]) < 1e-9 * max(1.0, abs(obs_o[-1, 0]))


@pytest.mark.gpu
@pytest.mark.parametrize("dims,beta", [((8, 8, 8), 0.693), ((16, 16, 4), 0.5), ((64, 64, 64), 0.693)])
def test_user_table_free_heisenberg(umc, oracle, lib, dims, beta):
    Lx, Ly, Lz = dims
    n = Lx * Ly * Lz
    pos = checker_position(Lx, Ly, Lz)
    ei, ej = cubic_edges(Lx, Ly, Lz)
    st, off, bonds, _ = oracle.pair_graph(n, *relabel_edges(ei, ej, pos))
    assert st == 0
    s = random_unit_vectors(n, 3, 5)
    sweeps = 2 if n > 100000 else 3
    for sweep in range(sweeps):
        cm = np.empty((n, 3))
        cm[pos] = s
        v_o, obs_o, margin = oracle.vector_metropolis(3, off, bonds, 1.0, beta, 0, 0.0, 6, sweep, 1, cm)
        flat = np.ascontiguousarray(s.reshape(-1))
        E = _d(0.0)
        _call(lib, lib.um_heisenberg_cubic(Lx, Ly, Lz, 1.0, beta, 6, sweep, 1, _p(flat), C.byref(E)))
        s = flat.reshape(n, 3)
        d = np.abs(s - v_o[pos]).max(axis=1)
        near = np.nonzero(np.abs(margin[pos]) < MARGIN)[0]
        bad = np.nonzero(d > TOL)[0]
        assert len(bad) <= 7 * len(near), (len(bad), len(near))
        assert abs(E.value - obs_o[0, 0]) < 1e-9 * n


@pytest.mark.gpu
def test_user_model_on_the_model_base(lib):
    """A model written on the device Model<T, Sites, Dof> base with a Field
    (Heisenberg8: the 8^3 table-free O(3) model's terms on the base's field)
    runs the same chain as the hand-written model: same state, same keys,
    bit-identical spins and energy after 5 sweeps from sweep 3."""
    s = random_unit_vectors(512, 3, 9)
    a = np.ascontiguousarray(s.reshape(-1)).copy()
    b = a.copy()
    Ea, Eb = _d(0.0), _d(0.0)
    _call(lib, lib.um_heisenberg_cubic(8, 8, 8, 1.0, 0.693, 6, 3, 5, _p(a), C.byref(Ea)))
    _call(lib, lib.um_heisenberg_cubic8_base(1.0, 0.693, 6, 3, 5, _p(b), C.byref(Eb)))
    assert not np.array_equal(a, s.reshape(-1))
    np.testing.assert_array_equal(a, b)
    assert Ea.value == Eb.value


def o3_wolff(lib, g, spins, beta, seed, flip0, n, sweeps=0):
    flat = np.ascontiguousarray(np.asarray(spins, np.float64).reshape(-1)).copy()
    sizes = np.zeros(max(n, 1), np.uint64)
    done = _u64(0)
    mean = _d(0.0)
    _call(lib, lib.um_o3_wolff(g._h, 1.0, beta, seed, flip0, n, sweeps, _p(flat),
                               sizes.ctypes.data_as(C.POINTER(_u64)), C.byref(done), C.byref(mean)))
    return flat.reshape(-1, 3), sizes[:n], done.value, mean.value


@pytest.mark.gpu
@pytest.mark.parametrize("L,beta,flips", [(8, 0.693, 12), (16, 0.693, 6), (12, 0.4, 10), (32, 0.75, 3)])
def test_user_wolff_flips(umc, oracle, lib, L, beta, flips):
    """Wolff<PairModel<Vec<3>, DotTerm<3>>, Sphere3>: every flip's cluster size
    equals the oracle's (driver.hpp:104-162 with the same keyed draws) and the
    field agrees to 1e-9, unless a bond test sat within 1e-9 of its threshold."""
    lib.um_o3_wolff.argtypes = [_vp, _d, _d, _u64, _u64, _u32, C.c_int, _dp, C.POINTER(_u64), C.POINTER(_u64),
                                C.POINTER(_d)]
    g = umc.cubic_lattice(L, L, L)
    n = L ** 3
    pos, doff, dbonds, key = device_csr(g)
    s = random_unit_vectors(n, 3, L)
    for f in range(flips):
        cm = np.empty((n, 3))
        cm[pos] = s
        v_o, sz_o, _, margin = oracle.vector_wolff(3, doff, dbonds, key, 1.0, beta, 21, f, 1, cm)
        s, sz, done, _ = o3_wolff(lib, g, s, beta, 21, f, 1)
        assert done == 1
        if margin[0] < MARGIN:
            continue
        assert sz[0] == sz_o[0], (f, sz, sz_o)
        assert np.abs(s - v_o[pos]).max() < TOL
    # several flips in one launch continue the same sequence
    a, sa, _, _ = o3_wolff(lib, g, s, beta, 21, 100, 5)
    b1, sb1, _, _ = o3_wolff(lib, g, s, beta, 21, 100, 2)
    b2, sb2, _, _ = o3_wolff(lib, g, b1, beta, 21, 102, 3)
    np.testing.assert_array_equal(a, b2)
    np.testing.assert_array_equal(sa, np.concatenate([sb1, sb2]))


@pytest.mark.gpu
def test_user_wolff_sweep_flips_until_the_lattice_is_covered(umc, oracle, lib):
    """Wolff::sweep (driver.hpp:163-173): flips until the flipped sites add up
    to the lattice; the number of flips and the field equal the oracle's."""
    lib.um_o3_wolff.argtypes = [_vp, _d, _d, _u64, _u64, _u32, C.c_int, _dp, C.POINTER(_u64), C.POINTER(_u64),
                                C.POINTER(_d)]
    L, beta = 10, 0.6
    g = umc.cubic_lattice(L, L, L)
    n = L ** 3
    pos, doff, dbonds, key = device_csr(g)
    s0 = random_unit_vectors(n, 3, 3)
    s, _, done, mean = o3_wolff(lib, g, s0, beta, 5, 0, 1, sweeps=1)
    cm = np.empty((n, 3))
    cm[pos] = s0
    touched, f, sizes = 0, 0, []
    while touched < n:
        cm, sz, _, margin = oracle.vector_wolff(3, doff, dbonds, key, 1.0, beta, 5, f, 1, cm)
        assert margin[0] >= MARGIN
        touched += int(sz[0])
        sizes.append(int(sz[0]))
        f += 1
    assert done == f
    assert abs(mean - np.mean(sizes)) < 1e-9
    assert np.abs(s - cm[pos]).max() < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("L,beta,tiled", [(16, 0.44, 0), (64, 0.3, 0), (48, 0.6, 0), (16, 0.44, 1), (64, 0.3, 1),
                                          (48, 0.6, 1), (200, 0.44, 1), (100, 0.5, 0)])
def test_user_ising_wolff_is_bit_exact(umc, oracle, lib, L, beta, tiled):
    """Wolff<PairModel<Spin, IsingBondTerm>, UpAxis> (int8 spins, int32 energy,
    FixedAxis): 20 flips in one launch equal the oracle's spins and cluster
    sizes bit for bit, with the global union-find alone (tiled 0) and with the
    shared-memory tiles first (tiled 1; 200^2 spans ten tiles)."""
    lib.um_ising_wolff.argtypes = [_vp, C.c_int32, _d, _u64, _u64, _u32, _vp, _vp, C.c_int]
    g = umc.square_lattice(L, L)
    n = L * L
    pos, doff, dbonds, key = device_csr(g)
    s0 = np.where(np.random.default_rng(L).random(n) < 0.5, 1, -1).astype(np.int8)
    s = s0.copy()
    sizes = np.zeros(20, np.uint64)
    _call(lib, lib.um_ising_wolff(g._h, 1, beta, 13, 7, 20, s.ctypes.data, sizes.ctypes.data, tiled))
    cm = np.empty(n, np.int8)
    cm[pos] = s0
    s_o, sz_o, _, _ = oracle.ising_wolff(doff, dbonds, key, 1, beta, 13, 7, 20, cm)
    np.testing.assert_array_equal(sizes, sz_o)
    np.testing.assert_array_equal(s, s_o[pos])


def lattice_csr(Lx, Ly, Lz):
    """RegularLattice's device numbering (colour-major checkerboard) and its
    bond rows in the order +x, -x, +y, -y, +z, -z over the extents above 1,
    with the Wolff keys k * degree + a from each bond's lower endpoint."""
    n = Lx * Ly * Lz
    s = np.arange(n)
    x, y, z = s % Lx, (s // Lx) % Ly, s // (Lx * Ly)
    pos = (((x + y + z) & 1) * (n // 2) + s // 2).astype(np.uint32)
    steps = [(1, 0, 0), (-1, 0, 0)]
    if Ly > 1:
        steps += [(0, 1, 0), (0, -1, 0)]
    if Lz > 1:
        steps += [(0, 0, 1), (0, 0, -1)]
    deg = len(steps)
    rows = np.empty((n, deg), np.uint32)
    for a, (dx, dy, dz) in enumerate(steps):
        t = (((z + dz) % Lz) * Ly + (y + dy) % Ly) * Lx + (x + dx) % Lx
        rows[pos, a] = pos[t]
    off = (np.arange(n + 1) * deg).astype(np.uint32)
    bonds = rows.reshape(-1)
    key = np.arange(n * deg, dtype=np.uint32)
    for k in range(n):
        for a in range(deg):
            j = rows[k, a]
            if j < k:
                back = np.nonzero(rows[j] == k)[0]
                assert len(back) == 1
                key[k * deg + a] = j * deg + back[0]
    return pos, off, bonds, key


def lattice_o3(lib, dims, spins, beta, seed, first, n, wolff):
    lib.um_lattice_o3.argtypes = [_u32, _u32, _u32, _d, _d, _u64, _u64, _u32, C.c_int, _dp, _vp]
    flat = np.ascontiguousarray(np.asarray(spins, np.float64).reshape(-1)).copy()
    sizes = np.zeros(max(n, 1), np.uint64)
    _call(lib, lib.um_lattice_o3(*dims, 1.0, beta, seed, first, n, wolff, _p(flat), sizes.ctypes.data))
    return flat.reshape(-1, 3), sizes[:n]


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(8, 8, 8), (16, 6, 1), (12, 4, 10)])
def test_user_term_on_table_free_lattice(umc, oracle, lib, dims):
    """LatticePairModel<Vec<3>, DotTerm<3>> over RegularLattice (no CSR on the
    device): Metropolis sweeps and Wolff flips equal the oracle on the same
    numbering and bond keys."""
    n = int(np.prod(dims))
    pos, off, bonds, key = lattice_csr(*dims)
    s = random_unit_vectors(n, 3, 8)
    for sweep in range(3):
        cm = np.empty((n, 3))
        cm[pos] = s
        v_o, _, margin = oracle.vector_metropolis(3, off, bonds, 1.0, 0.7, 0, 0.0, 17, sweep, 1, cm)
        s, _ = lattice_o3(lib, dims, s, 0.7, 17, sweep, 1, 0)
        d = np.abs(s - v_o[pos]).max(axis=1)
        assert (d > TOL).sum() <= 7 * (np.abs(margin) < MARGIN).sum()
    cm = np.empty((n, 3))
    cm[pos] = s
    v_o, sz_o, _, margin = oracle.vector_wolff(3, off, bonds, key, 1.0, 0.7, 23, 0, 6, cm)
    s2, sz = lattice_o3(lib, dims, s, 0.7, 23, 0, 6, 1)
    if margin.min() >= MARGIN:
        np.testing.assert_array_equal(sz, sz_o)
        assert np.abs(s2 - v_o[pos]).max() < TOL


@pytest.mark.gpu
def test_fp32_user_term_same_on_lattice_and_tables(umc, lib):
    """The FP32 O(3) user model of the bench runs the same chain on the
    table-free RegularLattice and on PairTables (same numbering and keys;
    only the neighbours' summation order differs), and its energy is finite
    and below the random start's."""
    vp = C.c_void_p
    lib.um_session_create.argtypes = [C.c_int, vp, _u32, _u32, _u32, _d, _d, _d, _u64, C.POINTER(vp)]
    lib.um_session_destroy.argtypes = [vp]
    lib.um_session_set_field.argtypes = [vp, vp]
    lib.um_session_get_field.argtypes = [vp, vp]
    lib.um_session_enqueue.argtypes = [vp, _u64]
    lib.um_session_stats.argtypes = [vp, C.POINTER(_u64), C.POINTER(_d), C.c_int]
    lib.um_session_energy.argtypes = [vp, C.POINTER(_d)]
    L, n = 16, 16 ** 3
    v0 = np.ascontiguousarray(random_unit_vectors(n, 3, 4), np.float32).reshape(-1)
    out, energies = [], []
    for kind in (1, 2):
        h = vp()
        _call(lib, lib.um_session_create(kind, None, L, L, L, 1.0, 0.693, 0.0, 3, C.byref(h)))
        try:
            _call(lib, lib.um_session_set_field(h, v0.ctypes.data))
            e0 = _d()
            _call(lib, lib.um_session_energy(h, C.byref(e0)))
            _call(lib, lib.um_session_enqueue(h, 5))
            cnt, ms = _u64(), _d()
            _call(lib, lib.um_session_stats(h, C.byref(cnt), C.byref(ms), 1))
            f = np.empty_like(v0)
            _call(lib, lib.um_session_get_field(h, f.ctypes.data))
            e = _d()
            _call(lib, lib.um_session_energy(h, C.byref(e)))
        finally:
            lib.um_session_destroy(h)
        out.append(f.reshape(n, 3))
        energies.append((e0.value, e.value))
    d = np.abs(out[0] - out[1]).max(axis=1)
    assert (d > 1e-4).sum() <= 20, (d > 1e-4).sum()
    for e0, e in energies:
        assert np.isfinite(e) and e < e0
    assert abs(np.linalg.norm(out[0], axis=1) - 1).max() < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("L", [64, 512])
def test_user_xy_energies_recorded_in_the_launch(umc, lib, L):
    """Metropolis::record_energy runs the sweeps in one launch and sums
    energy_at on the device after each: the same chain as sample() with a
    host observe after every sweep, and the same energies up to the
    summation order."""
    lib.um_xy_record.argtypes = [_vp, _d, _d, _d, _u64, _u64, _u32, _dp, _dp]
    g = umc.square_lattice(L, L)
    th0 = np.random.default_rng(L + 1).uniform(-np.pi, np.pi, L * L)
    a, ea, _ = xy_run(lib, g, th0, 1.1, 1.0, 12, 3, 6)
    b = th0.copy()
    eb = np.zeros(6)
    _call(lib, lib.um_xy_record(g._h, 1.0, 1.1, 1.0, 12, 3, 6, _p(b), _p(eb)))
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(eb, ea, rtol=1e-12, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,L,beta,width,sweeps", [("2d", 8, 2.0, 0.5, 3), ("4d", 4, 1.1, 0.7, 2),
                                                      ("4d", 6, 0.9, 1.0, 2), ("2d", 64, 1.5, 1.0, 2)])
def test_user_u1_on_table_free_plaquettes(umc, oracle, lib, kind, L, beta, width, sweeps):
    """LatticeCellModel over PlaquetteLattice (cells and incidence computed
    from the link index): the same chain as the oracle on the library's
    plaquette complex, relabelled by the library's link colouring."""
    lib.um_plaquette_u1.argtypes = [_u32, _u32, _d, _d, _d, _u64, _u64, _u32, _dp, _dp]
    dim = 2 if kind == "2d" else 4
    cc = umc.square_plaquettes(L) if kind == "2d" else umc.hypercubic_plaquettes(L)
    n = cc.sites()
    _, _, pos = cc.colouring()
    rcells = pos[cc.table()]
    inc = oracle.cell_incidence(n, rcells)[1:]
    th0 = np.random.default_rng(L + dim).uniform(-np.pi, np.pi, n)
    th = th0.copy()
    E = _d(0.0)
    _call(lib, lib.um_plaquette_u1(L, dim, beta, 1.0, width, 5, 0, sweeps, _p(th), C.byref(E)))
    cm = np.empty(n)
    cm[pos] = th0
    t_o, obs_o, _ = oracle.u1_metropolis(rcells, inc, beta, 1.0, width, 1, 5, 0, sweeps, cm)
    d = np.abs(np.angle(np.exp(1j * (th - t_o[pos]))))
    assert d.max() < TOL, d.max()
    assert abs(E.value - obs_o[-1, 0]) < 1e-9 * max(1.0, abs(obs_o[-1, 0]))


@pytest.mark.gpu
def test_device_header_barrier_wait_is_bounded(lib):
    """A block waiting at device.cuh's grid barrier for a block that never
    arrives gives up after its bounded wait, sets the status bit and returns
    (the kernel ends; nothing hangs)."""
    lib.um_barrier_selftest.argtypes = [C.POINTER(C.c_int)]
    out = C.c_int(0)
    _call(lib, lib.um_barrier_selftest(C.byref(out)))
    assert out.value == 1


@pytest.mark.gpu
@pytest.mark.parametrize("beta", [2.0, 4.0])
def test_user_su2_quaternion_gauge_model_matches_the_exact_2d_plaquette(lib, beta):
    """A gauge group given entirely by the user (SU(2) as unit quaternions, a
    Wilson plaquette term and a symmetric left-multiplication proposal) on the
    table-free 16 x 16 plaquettes: the mean plaquette recorded in the launch
    equals 2D lattice gauge theory's exact <(1/2) Tr U_p> = I_2(beta) / I_1(beta)
    within five binned standard errors."""
    from scipy.special import iv

    lib.um_su2_2d.argtypes = [_u32, _d, _d, _u64, _u32, _u32, _dp]
    n = 6000
    plaq = np.zeros(n)
    _call(lib, lib.um_su2_2d(16, beta, 1.0, 17, 500, n, _p(plaq)))
    exact = iv(2, beta) / iv(1, beta)
    bins = plaq[: n - n % 50].reshape(-1, 50).mean(axis=1)
    err = bins.std(ddof=1) / np.sqrt(len(bins))
    assert abs(plaq.mean() - exact) < 5 * err + 1e-4, (plaq.mean(), exact, err)


@pytest.mark.gpu
def test_user_xy_on_a_random_graph(umc, oracle, lib):
    """The generic kernel on an irregular, non-bipartite PairGraph (random
    edges, duplicates kept): the library's greedy colouring gives more than
    two classes, and every sweep still equals the oracle's on the relabelled
    graph."""
    rng = np.random.default_rng(31)
    n = 600
    ei = rng.integers(0, n, 2000)
    ej = (ei + rng.integers(1, n, 2000)) % n  # no self-loops
    g = umc.PairGraph(n, np.stack([ei, ej], axis=1).astype(np.uint32))
    ncol, _, pos = g.colouring()
    assert ncol > 2
    _, doff, dbonds, _ = device_csr(g)
    off_s, bonds_s = g.csr()
    th = rng.uniform(-np.pi, np.pi, n)
    for sweep in range(3):
        cm = np.empty(n)
        cm[pos] = th
        t_o, obs_o, margin = oracle.xy_metropolis(doff, dbonds, 1.0, 0.8, 1.2, 9, sweep, 1, cm)
        th, en, _ = xy_run(lib, g, th, 0.8, 1.2, 9, sweep, 1)
        d = np.abs(np.angle(np.exp(1j * (th - t_o[pos]))))
        near = np.nonzero(np.abs(margin[pos]) < MARGIN)[0]
        bad = set(np.nonzero(d > TOL)[0].tolist())
        assert bad <= set(near.tolist()) | _neighbours(off_s, bonds_s, near), sorted(bad)[:10]
        assert abs(en[0] - obs_o[0, 0]) < 1e-9 * n


@pytest.mark.gpu
@pytest.mark.parametrize("tiled", [0, 1])
def test_user_ising_wolff_on_a_random_graph(umc, oracle, lib, tiled):
    """The device Wolff on an irregular graph with duplicate edges (a bond
    listed twice is tested twice, as the reference's rows hold it twice), with
    and without the shared-memory tiles: spins and cluster sizes bit for bit
    against the oracle over 15 flips."""
    lib.um_ising_wolff.argtypes = [_vp, C.c_int32, _d, _u64, _u64, _u32, _vp, _vp, C.c_int]
    rng = np.random.default_rng(44)
    n = 9000  # three tiles of 4,096 reference sites
    ei = rng.integers(0, n, 20000)
    ej = (ei + rng.integers(1, 40, 20000)) % n  # mostly local bonds, some repeated
    g = umc.PairGraph(n, np.stack([ei, ej], axis=1).astype(np.uint32))
    pos, doff, dbonds, key = device_csr(g)
    s0 = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    s = s0.copy()
    sizes = np.zeros(15, np.uint64)
    _call(lib, lib.um_ising_wolff(g._h, 1, 0.35, 3, 0, 15, s.ctypes.data, sizes.ctypes.data, tiled))
    cm = np.empty(n, np.int8)
    cm[pos] = s0
    s_o, sz_o, _, _ = oracle.ising_wolff(doff, dbonds, key, 1, 0.35, 3, 0, 15, cm)
    np.testing.assert_array_equal(sizes, sz_o)
    np.testing.assert_array_equal(s, s_o[pos])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [1, 2])
def test_fp32_user_o3_term_per_sweep(umc, oracle, lib, kind):
    """The bench's FP32 user model (DotTermT<float, 3>, FP32 sphere proposal;
    kind 1 on the table-free lattice, kind 2 on CSR tables) against the FP64
    oracle, one sweep at a time from the same state: spins agree to 1e-5
    except at decisions within 1e-3 of their threshold and the sites next to
    them, as for the engine's FP32 chains."""
    vp = C.c_void_p
    lib.um_session_create.argtypes = [C.c_int, vp, _u32, _u32, _u32, _d, _d, _d, _u64, C.POINTER(vp)]
    lib.um_session_destroy.argtypes = [vp]
    lib.um_session_set_field.argtypes = [vp, vp]
    lib.um_session_get_field.argtypes = [vp, vp]
    lib.um_session_enqueue.argtypes = [vp, _u64]
    lib.um_session_stats.argtypes = [vp, C.POINTER(_u64), C.POINTER(_d), C.c_int]
    L, n = 8, 512
    pos, off, bonds, _ = lattice_csr(L, L, L)
    rows = {int(k): set(bonds[off[k]:off[k + 1]].tolist()) for k in range(n)}
    h = vp()
    _call(lib, lib.um_session_create(kind, None, L, L, L, 1.0, 0.693, 0.0, 7, C.byref(h)))
    try:
        s = np.ascontiguousarray(random_unit_vectors(n, 3, 12), np.float32)
        bad_total = 0
        for sweep in range(3):
            _call(lib, lib.um_session_set_field(h, s.ctypes.data))
            _call(lib, lib.um_session_enqueue(h, 1))
            cnt, ms = _u64(), _d()
            _call(lib, lib.um_session_stats(h, C.byref(cnt), C.byref(ms), 1))
            out = np.empty_like(s)
            _call(lib, lib.um_session_get_field(h, out.ctypes.data))
            cm = np.empty((n, 3))
            cm[pos] = s.astype(np.float64)
            v_o, _, margin = oracle.vector_metropolis(3, off, bonds, 1.0, 0.693, 0, 0.0, 7, sweep, 1, cm)
            d = np.abs(out.astype(np.float64) - v_o[pos]).max(axis=1)
            near = set(pos[np.nonzero(np.abs(margin[pos]) < 1e-3)[0]].tolist())  # device indices
            allowed = set(near)
            for k in near:
                allowed |= rows[k]
            bad = set(pos[np.nonzero(d > 1e-5)[0]].tolist())
            assert bad <= allowed, sorted(bad - allowed)[:10]
            bad_total += len(bad)
            s = out
        assert bad_total <= 20
    finally:
        lib.um_session_destroy(h)


# --------------------------------------- weighted models: PairGraph<double> payloads
def _device_payloads(g):
    """The bond payloads in the device rows' slot order (BondTables): rows in
    colour-major order, each row's slots in the reference row order."""
    off, _ = g.csr()
    _, _, pos = g.colouring()
    pay = g.payloads()
    return np.concatenate([pay[off[i]:off[i + 1]] for i in np.argsort(pos)])


def _weighted_graph(umc, kind):
    rng = np.random.default_rng(77)
    if kind == "random":
        n = 300
        e = rng.integers(0, n, (900, 2))
        e = e[e[:, 0] != e[:, 1]].astype(np.uint32)
        e = np.concatenate([e, e[:20]])  # duplicated bonds stay duplicated
    else:  # the reference graph test's 16 x 16 periodic lattice, random couplings
        n = 256
        e = np.stack(square_edges(16, 16), axis=1)
    c = rng.choice([-1.0, 1.0], len(e)) * rng.uniform(0.5, 1.5, len(e))
    return umc.PairGraph(n, e, payload=c), n


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["random", "square"])
def test_user_weighted_ising_metropolis_is_bit_exact(umc, oracle, lib, kind):
    """test/graph_check.cpp's IsingGraph as a user ModelLike on the device: double
    spins and the coupling carried by each bond of a PairGraph<double>
    (BondTables<double>::rows()), random +-J couplings.  30 sweeps equal the
    oracle's bit for bit (every decision is the FP64 test's), energies to 1e-12."""
    lib.um_weighted_ising.argtypes = [_vp, _d, _u64, _u64, _u32, C.c_int, C.c_int, _vp, _vp, _vp]
    g, n = _weighted_graph(umc, kind)
    pos, doff, dbonds, key = device_csr(g)
    cs = _device_payloads(g)
    s0 = np.where(np.random.default_rng(5).random(n) < 0.5, 1.0, -1.0)
    s = s0.copy()
    en = np.zeros(30)
    _call(lib, lib.um_weighted_ising(g._h, 0.45, 21, 4, 30, 0, 0, s.ctypes.data, en.ctypes.data, None))
    cm = np.empty(n)
    cm[pos] = s0
    s_o, E_o, margin = oracle.weighted_ising_metropolis(doff, dbonds, cs, 0.45, 21, 4, 30, cm)
    np.testing.assert_array_equal(s, s_o[pos])
    np.testing.assert_allclose(en, E_o, rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["random", "square"])
@pytest.mark.parametrize("tiled", [0, 1])
def test_user_weighted_ising_wolff_is_bit_exact(umc, oracle, lib, kind, tiled):
    """The same model under the device Wolff with the fixed axis: 25 flips, one
    launch each, equal the oracle's spins and cluster sizes bit for bit, with
    and without the shared-memory tiles; the bond tests read each bond's own
    coupling (energy_diff_bond = -c (p - s_j) s_i)."""
    lib.um_weighted_ising.argtypes = [_vp, _d, _u64, _u64, _u32, C.c_int, C.c_int, _vp, _vp, _vp]
    g, n = _weighted_graph(umc, kind)
    pos, doff, dbonds, key = device_csr(g)
    cs = _device_payloads(g)
    s0 = np.where(np.random.default_rng(6).random(n) < 0.5, 1.0, -1.0)
    s = s0.copy()
    sizes = np.zeros(25, np.uint64)
    en = np.zeros(25)
    _call(lib, lib.um_weighted_ising(g._h, 0.6, 33, 2, 25, 1, tiled, s.ctypes.data, en.ctypes.data,
                                     sizes.ctypes.data))
    cm = np.empty(n)
    cm[pos] = s0
    s_o, z_o, E_o = oracle.weighted_ising_wolff(doff, dbonds, key, cs, 0.6, 33, 2, 25, cm)
    np.testing.assert_array_equal(sizes, z_o)
    np.testing.assert_array_equal(s, s_o[pos])
    np.testing.assert_allclose(en, E_o, rtol=1e-12, atol=1e-12)
    assert sizes.max() > 1  # clusters grew


@pytest.mark.gpu
def test_builtin_models_refuse_weighted_graphs(umc):
    """As the reference's Ising and VectorSpin take PairGraph<> (no payload),
    the engine's built-in models refuse a graph with bond payloads."""
    g, _ = _weighted_graph(umc, "square")
    with pytest.raises(Exception, match="payload"):
        umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP, seed=1)
