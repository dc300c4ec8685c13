"""GPU parity for the spin models, through the C ABI.

Ising (Metropolis and Wolff) is compared bit-for-bit with the oracle: same
colour order, same keyed streams, integer thresholds.  The FP32 models are
compared one sweep (or one flip) at a time from an identical state: every site
must agree within TOL except sites whose accept decision the double-precision
oracle places within MARGIN of its threshold (and the neighbours they feed).

The engine takes every accept and activation decision as the FP64 test takes
it on its FP32 values (an FP32 test first, the FP64 one inside the FP32 test's
error band).  What remains between its decisions and the oracle's is the
rounding of the proposal itself: the FP32 candidate (hardware sine and cosine,
within about 4e-7 per component) against the oracle's FP64 one, which moves
log_p by at most beta |J| sum_c |h_c| 4e-7 < 3e-6 here (|h_c| <= 6), and the
FP32 Wolff axis, which moves 1 - exp(-x) by at most about 2e-6.  MARGIN is a few
times that.
"""
import numpy as np
import pytest

from helpers import checker_position, cubic_edges, random_unit_vectors, relabel_edges, square_edges

pytestmark = pytest.mark.gpu

TOL = 1e-5      # |component difference| allowed after one sweep (unit vectors / radians)
MARGIN = 2e-5   # |log u - log_p| (or |u - p| for Wolff) below which the FP32 candidate may flip a decision


def _engine_relabel(g):
    """The engine's colour-major relabelling of a PairGraph, for the oracle."""
    _, col, pos = g.colouring()
    return pos


def _oracle_csr(oracle, n, ei, ej):
    st, off, bonds, slot = oracle.pair_graph(n, ei, ej)
    assert st == 0
    return off, bonds, slot


def _graph_edges(umc, g):
    """Edge list of an engine graph, recovered from its CSR in edge order."""
    off, bonds = g.csr()
    ei, ej = [], []
    n = len(off) - 1
    for i in range(n):
        for a in range(off[i], off[i + 1]):
            if bonds[a] > i:
                ei.append(i)
                ej.append(bonds[a])
    return np.array(ei, np.uint32), np.array(ej, np.uint32)


# ----------------------------------------------------------------- Ising
def _ising_case(umc, oracle, g, ei, ej, J, beta, seed, sweeps, s0, sweep0=0):
    n = g.sites()
    pos = _engine_relabel(g)
    ri, rj = relabel_edges(ei, ej, pos)
    off, bonds, _ = _oracle_csr(oracle, n, ri, rj)
    cm0 = np.empty(n, np.int8)
    cm0[pos] = s0
    s_o, E_o, M_o = oracle.ising_metropolis(off, bonds, J, beta, seed, sweep0, sweeps, cm0)
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=J, proposal=umc.PROPOSAL_FLIP, seed=seed)
    ch.set_field(s0)
    ch.set_counters(sweep0, 0)
    rec = ch.metropolis(beta, sweeps)
    s_g = ch.get_field()
    np.testing.assert_array_equal(s_g, s_o[pos])
    np.testing.assert_array_equal(rec[:, 0], E_o)
    np.testing.assert_array_equal(rec[:, 1], M_o)
    assert ch.counters() == (sweep0 + sweeps, 0)
    return ch, rec


def test_ising_64x64_reference_config_bit_exact(umc, oracle):
    """Plain Metropolis, 2D Ising 64x64, J=1, beta=0.44, Flip, cold start, seed 1,
    2000 sweeps with energy and magnetisation recorded every sweep (packed
    checkerboard kernel)."""
    g = umc.square_lattice(64, 64)
    ei, ej = square_edges(64, 64)
    ch, rec = _ising_case(umc, oracle, g, ei, ej, 1, 0.44, 1, 2000, np.ones(4096, np.int8))
    assert rec[:, 7].sum() > 0  # proposals were accepted


@pytest.mark.parametrize("Lx,Ly", [(32, 2), (64, 6), (96, 32)])
def test_ising_packed_kernel_shapes(umc, oracle, Lx, Ly):
    g = umc.square_lattice(Lx, Ly)
    s0 = np.where(np.random.default_rng(Lx + Ly).random(Lx * Ly) < 0.5, -1, 1).astype(np.int8)
    _ising_case(umc, oracle, g, *square_edges(Lx, Ly), 1, 0.41, 17, 40, s0, sweep0=123)


@pytest.mark.parametrize("Lx,Ly,J,beta", [(6, 4, 1, 0.44), (2, 2, 1, 0.3), (2, 8, -1, 0.7), (10, 10, 2, 0.2)])
def test_ising_stencil_scalar_kernel(umc, oracle, Lx, Ly, J, beta):
    g = umc.square_lattice(Lx, Ly)
    s0 = np.where(np.random.default_rng(3).random(Lx * Ly) < 0.5, -1, 1).astype(np.int8)
    _ising_case(umc, oracle, g, *square_edges(Lx, Ly), J, beta, 5, 60, s0)


@pytest.mark.parametrize("Lx,Ly", [(3, 3), (5, 7), (1, 6), (3, 1)])
def test_ising_odd_lattices_csr(umc, oracle, Lx, Ly):
    g = umc.square_lattice(Lx, Ly)
    s0 = np.where(np.random.default_rng(4).random(Lx * Ly) < 0.5, -1, 1).astype(np.int8)
    _ising_case(umc, oracle, g, *square_edges(Lx, Ly), 1, 0.4, 9, 50, s0)


def test_ising_3d_and_random_graph(umc, oracle):
    g = umc.cubic_lattice(4, 4, 4)
    s0 = np.where(np.random.default_rng(5).random(64) < 0.5, -1, 1).astype(np.int8)
    _ising_case(umc, oracle, g, *cubic_edges(4, 4, 4), 1, 0.22, 3, 30, s0)
    rng = np.random.default_rng(6)
    e = rng.integers(0, 100, (260, 2))
    e = e[e[:, 0] != e[:, 1]].astype(np.uint32)
    g = umc.PairGraph(100, e)
    s0 = np.where(rng.random(100) < 0.5, -1, 1).astype(np.int8)
    _ising_case(umc, oracle, g, e[:, 0].copy(), e[:, 1].copy(), 1, 0.3, 8, 30, s0)


def test_ising_directed_graph(umc, oracle):
    rng = np.random.default_rng(7)
    e = rng.integers(0, 40, (120, 2))
    e = e[e[:, 0] != e[:, 1]].astype(np.uint32)
    g = umc.PairGraph(40, e, symmetric=False)
    pos = _engine_relabel(g)
    ri, rj = relabel_edges(e[:, 0].copy(), e[:, 1].copy(), pos)
    st, off, bonds, _ = oracle.pair_graph(40, ri, rj, symmetric=False)
    s0 = np.where(rng.random(40) < 0.5, -1, 1).astype(np.int8)
    cm0 = np.empty(40, np.int8)
    cm0[pos] = s0
    s_o, E_o, M_o = oracle.ising_metropolis(off, bonds, 1, 0.5, 2, 0, 20, cm0)
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP, seed=2)
    ch.set_field(s0)
    rec = ch.metropolis(0.5, 20)
    np.testing.assert_array_equal(ch.get_field(), s_o[pos])
    np.testing.assert_array_equal(rec[:, 0], E_o)
    np.testing.assert_array_equal(rec[:, 1], M_o)


def _ising_wolff_case(umc, oracle, g, ei, ej, J, beta, seed, flips, s0):
    n = g.sites()
    pos = _engine_relabel(g)
    ri, rj = relabel_edges(ei, ej, pos)
    off, bonds, slot = _oracle_csr(oracle, n, ri, rj)
    cm0 = np.empty(n, np.int8)
    cm0[pos] = s0
    s_o, z_o, E_o, M_o = oracle.ising_wolff(off, bonds, slot, J, beta, seed, 0, flips, cm0)
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=J, proposal=umc.PROPOSAL_FLIP,
                   wolff_axis=umc.AXIS_FIXED, seed=seed)
    ch.set_field(s0)
    sizes, rec = ch.wolff(beta, flips)
    np.testing.assert_array_equal(sizes, z_o)
    np.testing.assert_array_equal(ch.get_field(), s_o[pos])
    np.testing.assert_array_equal(rec[:, 0], E_o)
    np.testing.assert_array_equal(rec[:, 1], M_o)
    np.testing.assert_array_equal(rec[:, 7], z_o)
    f, ssum = ch.wolff_stats()
    assert f == flips and ssum == z_o.sum()
    return ch


@pytest.mark.parametrize("L,beta", [(16, 0.44), (64, 0.44), (8, 0.2), (2, 0.6)])
def test_ising_wolff_bit_exact(umc, oracle, L, beta):
    g = umc.square_lattice(L, L)
    s0 = np.where(np.random.default_rng(L).random(L * L) < 0.5, -1, 1).astype(np.int8)
    _ising_wolff_case(umc, oracle, g, *square_edges(L, L), 1, beta, 3, 200, s0)


def test_ising_wolff_odd_and_random_graph(umc, oracle):
    g = umc.square_lattice(5, 3)
    s0 = np.ones(15, np.int8)
    _ising_wolff_case(umc, oracle, g, *square_edges(5, 3), 1, 0.5, 4, 100, s0)
    rng = np.random.default_rng(8)
    e = rng.integers(0, 60, (150, 2))
    e = e[e[:, 0] != e[:, 1]].astype(np.uint32)
    g = umc.PairGraph(60, e)
    s0 = np.where(rng.random(60) < 0.5, -1, 1).astype(np.int8)
    _ising_wolff_case(umc, oracle, g, e[:, 0].copy(), e[:, 1].copy(), 2, 0.3, 6, 100, s0)


def test_ising_wolff_then_metropolis_hybrid(umc, oracle):
    L = 32
    g = umc.square_lattice(L, L)
    ei, ej = square_edges(L, L)
    pos = _engine_relabel(g)
    ri, rj = relabel_edges(ei, ej, pos)
    off, bonds, slot = _oracle_csr(oracle, L * L, ri, rj)
    s = np.ones(L * L, np.int8)
    sizes_o, E_o = [], []
    for k in range(30):
        s, z, _, _ = oracle.ising_wolff(off, bonds, slot, 1, 0.44, 7, k, 1, s)
        s, E, _ = oracle.ising_metropolis(off, bonds, 1, 0.44, 7, k, 1, s)
        sizes_o.append(z[0])
        E_o.append(E[0])
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP,
                   wolff_axis=umc.AXIS_FIXED, seed=7)
    sizes, rec = ch.hybrid(0.44, 30)
    np.testing.assert_array_equal(sizes, sizes_o)
    np.testing.assert_array_equal(rec[:, 0], E_o)
    np.testing.assert_array_equal(ch.get_field(), s[pos])


# ------------------------------------------------------------ FP32 models
def _neighbours(off, bonds, idx):
    out = set()
    for i in idx:
        out.update(bonds[off[i]:off[i + 1]].tolist())
    return out


def _compare_sweep(state_gpu, state_ora, margins, off, bonds, tol=TOL):
    """Sites off by more than tol must be near-margin sites or their neighbours."""
    diff = np.abs(state_gpu - state_ora).reshape(len(margins), -1).max(axis=1)
    bad = np.nonzero(diff > tol)[0]
    near = np.nonzero(np.abs(margins) < MARGIN)[0]
    allowed = set(near.tolist()) | _neighbours(off, bonds, near)
    assert set(bad.tolist()) <= allowed, (bad, near, diff[bad])
    return len(bad)


def _vector_setup(umc, oracle, g, ei, ej):
    n = g.sites()
    pos = _engine_relabel(g)
    ri, rj = relabel_edges(ei, ej, pos)
    off, bonds, slot = _oracle_csr(oracle, n, ri, rj)
    return pos, off, bonds, slot


@pytest.mark.parametrize("N,prop,dims", [(3, 0, (8, 8, 8)), (3, 1, (8, 8, 8)), (2, 1, (16, 16, 1)),
                                         (4, 0, (6, 6, 1)), (1, 0, (8, 8, 1)), (3, 0, (5, 5, 1)),
                                         (2, 0, (4, 2, 6))])
def test_vector_metropolis_per_sweep(umc, oracle, N, prop, dims):
    Lx, Ly, Lz = dims
    n = Lx * Ly * Lz
    g = umc.cubic_lattice(Lx, Ly, Lz) if Lz > 1 else umc.square_lattice(Lx, Ly)
    ei, ej = cubic_edges(Lx, Ly, Lz)
    pos, off, bonds, _ = _vector_setup(umc, oracle, g, ei, ej)
    kind = umc.PROPOSAL_SPHERE if prop == 0 else umc.PROPOSAL_ROTATION
    ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=N, coupling=1.0, proposal=kind, width=0.6, seed=5)
    v = random_unit_vectors(n, N, 3).astype(np.float32)
    ch.set_field(v)
    mism = 0
    for sweep in range(4):
        state = ch.get_field().reshape(n, N)
        cm = np.empty((n, N))
        cm[pos] = state
        v_o, obs_o, margin = oracle.vector_metropolis(N, off, bonds, 1.0, 0.693, prop, 0.6, 5, sweep, 1, cm)
        rec = ch.metropolis(0.693, 1)
        got = ch.get_field().reshape(n, N)
        mism += _compare_sweep(got, v_o[pos], margin[pos], *_site_csr(umc, g))
        # the fused FP64 record equals the observables of the new state
        e_true = _vector_energy(g, got.astype(np.float64))
        assert abs(rec[0, 0] - e_true) < 1e-5 * max(1.0, abs(e_true))
        np.testing.assert_allclose(rec[0, 1:1 + N], got.astype(np.float64).sum(axis=0), rtol=0, atol=1e-4)
    assert mism <= max(2, n // 50)


def _site_csr(umc, g):
    off, bonds = g.csr()
    return off, bonds


def _vector_energy(g, s):
    off, bonds = g.csr()
    e = 0.0
    for i in range(len(off) - 1):
        for a in range(off[i], off[i + 1]):
            e += -1.0 * float(np.dot(s[i], s[bonds[a]]))
    return 0.5 * e


@pytest.mark.parametrize("L", [8, 16, 24])
def test_vector_wolff_per_flip(umc, oracle, L):
    """One O(3) Wolff flip at a time from an identical state, on one 8^3 tile
    and on 8 and 27 tiles (the tile-crossing bonds of the fused kernel)."""
    g = umc.cubic_lattice(L, L, L)
    n = L**3
    ei, ej = cubic_edges(L, L, L)
    pos, off, bonds, slot = _vector_setup(umc, oracle, g, ei, ej)
    ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE,
                   wolff_axis=umc.AXIS_SPHERE, seed=9)
    v0 = random_unit_vectors(n, 3, 4)
    if L > 8:  # a partly ordered start: clusters span many tiles
        v0 = v0 * 0.8 + np.array([0.0, 0.0, 1.0])
        v0 /= np.linalg.norm(v0, axis=1, keepdims=True)
    ch.set_field(v0.astype(np.float32))
    checked, big = 0, 0
    for f in range(40):
        state = ch.get_field().reshape(n, 3)
        cm = np.empty((n, 3))
        cm[pos] = state
        v_o, z_o, obs_o, margin = oracle.vector_wolff(3, off, bonds, slot, 1.0, 0.693, 9, f, 1, cm)
        sizes, rec = ch.wolff(0.693, 1)
        got = ch.get_field().reshape(n, 3)
        if margin[0] < MARGIN:
            continue  # an activation decision sat on its threshold: resync
        checked += 1
        big += int(z_o[0] > 512)
        assert sizes[0] == z_o[0]
        np.testing.assert_allclose(got, v_o[pos], rtol=0, atol=TOL)
    assert checked >= 30
    assert L == 8 or big >= 5  # clusters beyond one tile were compared


def test_xy_angle_per_sweep(umc, oracle):
    L = 16
    g = umc.square_lattice(L, L)
    n = L * L
    ei, ej = square_edges(L, L)
    pos, off, bonds, _ = _vector_setup(umc, oracle, g, ei, ej)
    ch = umc.Chain(umc.MODEL_XY_ANGLE, graph=g, coupling=1.0, proposal=umc.PROPOSAL_U1SHIFT, width=1.0, seed=4)
    th = np.random.default_rng(1).uniform(-np.pi, np.pi, n).astype(np.float32)
    ch.set_field(th)
    mism = 0
    for sweep in range(4):
        state = ch.get_field().astype(np.float64)
        cm = np.empty(n)
        cm[pos] = state
        t_o, obs_o, margin = oracle.xy_metropolis(off, bonds, 1.0, 1.1, 1.0, 4, sweep, 1, cm)
        rec = ch.metropolis(1.1, 1)
        got = ch.get_field().astype(np.float64)
        d = np.abs(np.angle(np.exp(1j * (got - t_o[pos]))))
        sel = d > TOL * 4
        near = np.abs(margin[pos]) < MARGIN
        off_s, bonds_s = g.csr()
        allowed = set(np.nonzero(near)[0].tolist()) | _neighbours(off_s, bonds_s, np.nonzero(near)[0])
        assert set(np.nonzero(sel)[0].tolist()) <= allowed
        mism += int(sel.sum())
        np.testing.assert_allclose(rec[0, 0], obs_o[0, 0], rtol=1e-4, atol=1e-3)
    assert mism <= 4


def test_large_lattice_observables_are_consistent(umc):
    """Size-independent checks on a 2048^2 Ising lattice and a 64^3 O(3)
    lattice: the fused per-sweep record equals a separate full recomputation
    and the magnetisation equals the sum of the field."""
    g = umc.square_lattice(2048, 2048)
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP, seed=3)
    ch.randomize(11)
    rec = ch.metropolis(0.44, 5)
    obs = ch.observe()
    assert rec[-1, 0] == obs[0] and rec[-1, 1] == obs[1]
    s = ch.get_field()
    assert rec[-1, 1] == s.astype(np.int64).sum()
    assert set(np.unique(s).tolist()) <= {-1, 1}
    g3 = umc.cubic_lattice(64, 64, 64)
    ch3 = umc.Chain(umc.MODEL_VECTOR, graph=g3, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE,
                    wolff_axis=umc.AXIS_SPHERE, seed=1)
    ch3.randomize(1)
    sizes, rec = ch3.hybrid(0.693, 10)
    obs = ch3.observe()
    assert abs(rec[-1, 0] - obs[0]) < 1e-6 * abs(obs[0]) + 1e-6
    v = ch3.get_field().astype(np.float64)
    assert np.abs(np.linalg.norm(v, axis=1) - 1).max() < 1e-5
    np.testing.assert_allclose(rec[-1, 1:4], v.sum(axis=0), atol=1e-2)
    assert (sizes >= 1).all()


def test_randomize_is_keyed_and_deterministic(umc, oracle):
    g = umc.square_lattice(8, 8)
    ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE, seed=1)
    ch.randomize(42)
    a = ch.get_field()
    ch.randomize(42)
    np.testing.assert_array_equal(a, ch.get_field())
    # site i draws UniformSphereN<3> from key (42, 0, tag 3, i)
    from oracle.oracle import TAG_INIT
    for i in [0, 5, 63]:
        k = oracle.key_draws(42, 0, TAG_INIT, i, 2)
        z = 2.0 * k[0] * 2.0**-32 - 1.0
        phi = 2 * np.pi * k[1] * 2.0**-32
        r = np.sqrt(1 - z * z)
        np.testing.assert_allclose(a[i], [r * np.cos(phi), r * np.sin(phi), z], atol=2e-6)


def test_counters_key_the_streams(umc):
    """A chain is a pure function of (field, seed, counters): replaying from the
    same state and counters reproduces the trajectory exactly."""
    g = umc.cubic_lattice(8, 8, 8)
    ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE,
                   wolff_axis=umc.AXIS_SPHERE, seed=77)
    ch.randomize(5)
    ch.hybrid(0.7, 3)
    snap = ch.get_field()
    sw, fl = ch.counters()
    _, rec1 = ch.hybrid(0.7, 5)
    end1 = ch.get_field()
    ch.set_field(snap)
    ch.set_counters(sw, fl)
    _, rec2 = ch.hybrid(0.7, 5)
    np.testing.assert_array_equal(rec1, rec2)
    np.testing.assert_array_equal(end1, ch.get_field())


def test_invalid_combinations_are_rejected(umc):
    g = umc.square_lattice(4, 4)
    with pytest.raises(umc.UmcError):
        umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_SPHERE)
    with pytest.raises(ValueError):
        umc.Chain(umc.MODEL_ISING, graph=g, coupling=0.5)
    ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE)
    with pytest.raises(umc.UmcError):
        ch.wolff(0.5, 1)  # no axis configured
    with pytest.raises(ValueError):
        ch.metropolis(float("nan"), 1)


@pytest.mark.parametrize("dims,N,prop", [((16, 16, 16), 3, "sphere"), ((32, 32, 1), 2, "rotation"),
                                         ((8, 8, 8), 4, "sphere"), ((6, 4, 2), 3, "rotation"),
                                         ((64, 64, 64), 3, "sphere"), ((12, 10, 14), 3, "sphere"),
                                         ((40, 18, 1), 2, "sphere"), ((24, 8, 2), 1, "sphere")])
def test_fused_step_matches_multikernel(umc, dims, N, prop):
    """The one-kernel step (cooperative, grid barrier) and the five-kernel path
    produce the same field, cluster sizes and accept counts."""
    g = umc.cubic_lattice(*dims) if dims[2] > 1 else umc.square_lattice(dims[0], dims[1])
    kind = umc.PROPOSAL_SPHERE if prop == "sphere" else umc.PROPOSAL_ROTATION
    chains = []
    for fused in (True, False):
        ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=N, coupling=1.0, proposal=kind, width=0.8,
                       wolff_axis=umc.AXIS_SPHERE, seed=21)
        ch.set_fused(fused)
        ch.randomize(4)
        chains.append(ch)
    out = []
    for ch in chains:
        ch.kernel_stats(reset=True)
        s1, r1 = ch.hybrid(0.693, 12)
        r2 = ch.metropolis(0.693, 5)
        s3, r3 = ch.wolff(0.693, 5)
        out.append((s1, r1, r2, s3, r3, ch.get_field(), ch.kernel_stats()))
    a, b = out
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[3], b[3])
    np.testing.assert_array_equal(a[5], b[5])
    for ra, rb in ((a[1], b[1]), (a[2], b[2]), (a[4], b[4])):
        np.testing.assert_array_equal(ra[:, 7], rb[:, 7])
        np.testing.assert_allclose(ra[:, :5], rb[:, :5], rtol=1e-9, atol=1e-6)
    assert a[6]["fused"][0] == 12 + 5 + 5 and a[6]["metropolis"][0] == 0
    assert b[6]["fused"][0] == 0


@pytest.mark.parametrize("model", ["o3", "ising"])
def test_async_upload_and_record_streaming_match_the_synchronous_path(umc, model):
    """Uploads queued back to back (two staging buffers, a copy stream) and
    records streamed to host memory give the same records, cluster sizes and
    final field as set_field + hybrid run per configuration."""
    rng = np.random.default_rng(3)
    if model == "o3":
        g = umc.cubic_lattice(16, 16, 16)
        mk = lambda: umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0,
                               proposal=umc.PROPOSAL_SPHERE, wolff_axis=umc.AXIS_SPHERE, seed=9)
        fields = []
        for _ in range(5):
            v = rng.normal(size=(g.sites(), 3))
            fields.append((v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32))
        beta = 0.693
    else:
        g = umc.square_lattice(64, 64)
        mk = lambda: umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP,
                               wolff_axis=umc.AXIS_FIXED, seed=9)
        fields = [np.where(rng.random(g.sites()) < 0.5, -1, 1).astype(np.int8) for _ in range(5)]
        beta = 0.44
    a, b = mk(), mk()
    sa, ra = [], []
    for f in fields:
        a.set_field(f)
        s_, r_ = a.hybrid(beta, 3)
        sa.append(s_)
        ra.append(r_)
    b.set_record_streaming(True)
    for f in fields:
        b.upload_async(np.ascontiguousarray(f))
        b.enqueue_hybrid(beta, 3)
    rb, sb = b.fetch(64)
    np.testing.assert_array_equal(np.concatenate(ra), rb)
    np.testing.assert_array_equal(np.concatenate(sa), sb)
    np.testing.assert_array_equal(a.get_field(), b.get_field())
    # streaming off again: the synchronous path keeps working
    b.set_record_streaming(False)
    b.set_field(fields[0])
    a.set_field(fields[0])
    np.testing.assert_array_equal(a.hybrid(beta, 2)[1], b.hybrid(beta, 2)[1])
