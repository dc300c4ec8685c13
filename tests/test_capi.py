"""The C ABI library on a host without a GPU: it loads, exports every symbol the
header declares, builds the reference's tables identically, and fails loudly
(no CPU fallback) when asked to create a chain."""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import checker_position, cubic_edges, link_class_position, square_edges

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(umc_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol(umc):
    names = _declared_symbols()
    assert len(names) > 30
    missing = [n for n in sorted(names) if not hasattr(umc.lib, n)]
    assert not missing, missing


def test_abi_version(umc):
    assert umc.lib.umc_abi_version() == 2


@pytest.mark.parametrize("Lx,Ly", [(1, 1), (1, 4), (2, 2), (4, 4), (3, 5), (8, 6)])
def test_square_lattice_matches_oracle(umc, oracle, Lx, Ly):
    g = umc.square_lattice(Lx, Ly)
    off, bonds = g.csr()
    _, ei, ej = oracle.square_edges(Lx, Ly)
    _, off2, bonds2, _ = oracle.pair_graph(Lx * Ly, ei, ej)
    np.testing.assert_array_equal(off, off2)
    np.testing.assert_array_equal(bonds, bonds2)


def test_square_lattice_matches_reference(umc, golden):
    for Lx, Ly in [(1, 1), (1, 4), (2, 2), (4, 4), (3, 5)]:
        off, bonds = umc.square_lattice(Lx, Ly).csr()
        np.testing.assert_array_equal(off, golden[f"square_{Lx}x{Ly}_off"])
        np.testing.assert_array_equal(bonds, golden[f"square_{Lx}x{Ly}_bonds"])


def test_cubic_lattice_matches_edge_list(umc, oracle):
    g = umc.cubic_lattice(4, 2, 6)
    off, bonds = g.csr()
    ei, ej = cubic_edges(4, 2, 6)
    _, off2, bonds2, _ = oracle.pair_graph(48, ei, ej)
    np.testing.assert_array_equal(off, off2)
    np.testing.assert_array_equal(bonds, bonds2)


def test_graph_errors_mirror_reference_exceptions(umc):
    with pytest.raises(ValueError):
        umc.PairGraph(2, [[0, 0]])  # self-loop: std::invalid_argument
    with pytest.raises(IndexError):
        umc.PairGraph(2, [[0, 2]])  # std::out_of_range
    with pytest.raises(OverflowError):
        umc.PairGraph(2**32 + 1, [])  # std::overflow_error
    with pytest.raises(ValueError):
        umc.square_lattice(0, 3)
    with pytest.raises(ValueError):
        umc.hypercubic_plaquettes(0)
    with pytest.raises(IndexError):
        umc.CellComplex(3, [[0, 1, 2, 3]])
    g = umc.PairGraph(2, [[0, 1], [0, 1]])
    assert g.degree(0) == 2  # duplicates kept
    g = umc.PairGraph(3, [])
    assert g.sites() == 3 and g.degree(1) == 0
    g = umc.PairGraph(2, [[0, 1]], symmetric=False)
    assert g.degree(0) == 1 and g.degree(1) == 0


@pytest.mark.parametrize("dims", [(8, 8, 1), (2, 2, 1), (6, 4, 1), (4, 4, 4), (2, 6, 8)])
def test_even_lattices_use_the_checkerboard(umc, dims):
    g = umc.cubic_lattice(*dims) if dims[2] > 1 else umc.square_lattice(dims[0], dims[1])
    nc, col, pos = g.colouring()
    assert nc == 2
    np.testing.assert_array_equal(pos, checker_position(*dims))


@pytest.mark.parametrize("Lx,Ly", [(3, 3), (5, 4), (3, 7)])
def test_odd_lattices_get_a_valid_colouring(umc, oracle, Lx, Ly):
    g = umc.square_lattice(Lx, Ly)
    nc, col, pos = g.colouring()
    off, bonds = g.csr()
    assert nc >= 3 and oracle.check_colouring(off, bonds, col)
    assert sorted(pos) == list(range(Lx * Ly))
    # colour-major: classes contiguous, ascending site id inside a class
    order = np.argsort(pos)
    assert (np.diff(col[order]) >= 0).all()
    for c in range(nc):
        sites = order[col[order] == c]
        assert (np.diff(sites) > 0).all()


def test_random_graph_colouring_is_valid(umc, oracle):
    rng = np.random.default_rng(2)
    n = 200
    e = rng.integers(0, n, (700, 2))
    e = e[e[:, 0] != e[:, 1]]
    g = umc.PairGraph(n, e)
    nc, col, pos = g.colouring()
    off, bonds = g.csr()
    assert oracle.check_colouring(off, bonds, col)
    gd = umc.PairGraph(n, e, symmetric=False)
    _, cold, _ = gd.colouring()
    sym_off, sym_b = umc.PairGraph(n, e).csr()
    assert oracle.check_colouring(sym_off, sym_b, cold)


def test_hypercubic_matches_reference(umc, golden):
    c = umc.hypercubic_plaquettes(2)
    np.testing.assert_array_equal(c.table(), golden["hyper2_cells"])
    off, ic, iw = c.incidence()
    np.testing.assert_array_equal(off, golden["hyper2_off"])
    np.testing.assert_array_equal(ic, golden["hyper2_inc_cell"])
    np.testing.assert_array_equal(iw, golden["hyper2_inc_which"])


@pytest.mark.parametrize("L,dim", [(2, 4), (4, 4), (4, 2), (8, 2)])
def test_plaquette_complexes_use_direction_parity_classes(umc, oracle, L, dim):
    c = umc.hypercubic_plaquettes(L) if dim == 4 else umc.square_plaquettes(L)
    nc, col, pos = c.colouring()
    assert nc == 2 * dim
    np.testing.assert_array_equal(pos, link_class_position(L, dim))
    assert oracle.check_cell_colouring(c.sites(), c.table(), col)


def test_odd_plaquette_complex_colouring_is_valid(umc, oracle):
    c = umc.hypercubic_plaquettes(3)
    nc, col, _ = c.colouring()
    assert oracle.check_cell_colouring(c.sites(), c.table(), col)
    c2 = umc.square_plaquettes(5)
    _, col2, _ = c2.colouring()
    assert oracle.check_cell_colouring(c2.sites(), c2.table(), col2)


def test_chain_fails_loudly_without_gpu(umc):
    if umc.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(umc.UmcError) as e:
        umc.Chain(umc.MODEL_ISING, graph=umc.square_lattice(4, 4), coupling=1)
    assert e.value.code == umc.ERR_CUDA


def test_ising_thresholds_pin_the_reference_accept_rule():
    """accept iff draw <= tm1 reproduces log(k 2^-32) < -beta dE exactly."""
    import math

    for beta, dE in [(0.44, 4), (0.44, 8), (0.3, 4), (1.7, 12), (0.01, 2)]:
        log_p = -beta * dE + 0.0
        lo, hi = 0, 1 << 32
        while hi - lo > 1:
            mid = (lo + hi) // 2
            if math.log(mid * 2.0**-32) < log_p:
                lo = mid
            else:
                hi = mid
        assert math.log(lo * 2.0**-32) < log_p
        assert not math.log((lo + 1) * 2.0**-32) < log_p


# ------------------------------------------------------ bond payloads (PairGraph<P>)
def test_payload_graph_copies_edge_payloads_into_both_slots(umc):
    """PairGraph<double>(n, edges): every slot carries its edge's payload
    (lattice/pair_graph.hpp:77-81), duplicates and the directed form included;
    the CSR itself is the NoPayload graph's."""
    from helpers import slot_edges

    rng = np.random.default_rng(9)
    e = rng.integers(0, 30, (80, 2))
    e = e[e[:, 0] != e[:, 1]].astype(np.uint32)
    e = np.concatenate([e, e[:3]])  # duplicated edges stay duplicated
    c = rng.normal(size=len(e))
    for symmetric in (True, False):
        g = umc.PairGraph(30, e, symmetric=symmetric, payload=c)
        g0 = umc.PairGraph(30, e, symmetric=symmetric)
        off, bonds = g.csr()
        off0, bonds0 = g0.csr()
        np.testing.assert_array_equal(off, off0)
        np.testing.assert_array_equal(bonds, bonds0)
        slot = slot_edges(off, e[:, 0], e[:, 1], symmetric)
        np.testing.assert_array_equal(g.slot_edges(), slot)
        np.testing.assert_array_equal(g.payloads(), c[slot])
    # a record of several values per edge (a structured payload)
    rec = rng.normal(size=(len(e), 3)).astype(np.float32)
    g = umc.PairGraph(30, e, payload=rec)
    np.testing.assert_array_equal(g.payloads(), rec[slot_edges(g.csr()[0], e[:, 0], e[:, 1])])
    assert umc.lib.umc_graph_payload_bytes(g._h) == 12
    assert umc.lib.umc_graph_payload_bytes(umc.PairGraph(30, e)._h) == 0


def test_payload_graph_errors(umc):
    e = np.array([[0, 1], [1, 2]], np.uint32)
    ei, ej = np.ascontiguousarray(e[:, 0]), np.ascontiguousarray(e[:, 1])
    h = umc._vp()
    pay = np.zeros(2 * 300, np.uint8)
    for nbytes in (0, 257):
        rc = umc.lib.umc_graph_create_payload(3, ei.ctypes.data, ej.ctypes.data, 2, 1, pay.ctypes.data, nbytes,
                                              ctypes.byref(h))
        assert rc == umc.ERR_INVALID_ARGUMENT
    rc = umc.lib.umc_graph_create_payload(3, ei.ctypes.data, ej.ctypes.data, 2, 1, None, 8, ctypes.byref(h))
    assert rc == umc.ERR_INVALID_ARGUMENT
    # the reference's construction rules still apply
    with pytest.raises(ValueError):
        umc.PairGraph(3, [[0, 0]], payload=np.ones(1))
    with pytest.raises(IndexError):
        umc.PairGraph(3, [[0, 5]], payload=np.ones(1))
    with pytest.raises(ValueError):
        umc.PairGraph(3, e, payload=np.ones(3))  # one record per edge
    with pytest.raises(ValueError):
        umc.PairGraph(3, e).payloads()


def test_slab_descriptions_are_checked(umc):
    """umc_slab_create refuses what the decomposition cannot run, before any
    device work: odd or unit extents, planes outside the lattice, other
    models and proposals."""
    def create(**kw):
        d = umc.SlabDesc()
        d.model, d.components, d.Lx, d.Ly, d.Lz = umc.MODEL_ISING, 1, 8, 8, 1
        d.first_plane, d.planes, d.coupling, d.proposal, d.seed = 0, 4, 1.0, umc.PROPOSAL_FLIP, 1
        for k, v in kw.items():
            setattr(d, k, v)
        h = umc._vp()
        rc = umc.lib.umc_slab_create(ctypes.byref(d), ctypes.byref(h))
        if rc == umc.OK:
            umc.lib.umc_slab_destroy(h)
        return rc

    assert create(Lx=7) == umc.ERR_INVALID_ARGUMENT
    assert create(Ly=1) == umc.ERR_INVALID_ARGUMENT
    assert create(Lz=3) == umc.ERR_INVALID_ARGUMENT
    assert create(first_plane=6, planes=3) == umc.ERR_OUT_OF_RANGE
    assert create(planes=0) == umc.ERR_OUT_OF_RANGE
    assert create(coupling=0.5) == umc.ERR_INVALID_ARGUMENT
    assert create(model=umc.MODEL_U1) == umc.ERR_UNSUPPORTED
    assert create(model=umc.MODEL_VECTOR, components=3, proposal=umc.PROPOSAL_FLIP) == umc.ERR_UNSUPPORTED
    assert create(model=umc.MODEL_VECTOR, components=5, proposal=umc.PROPOSAL_SPHERE) == umc.ERR_UNSUPPORTED


def test_gauge_slab_descriptions_are_checked(umc):
    """umc_gslab_create refuses what the decomposition cannot run, before any
    device work: missing tables or owners, a rank outside the world, no hits,
    non-finite couplings, other models and SU(N) beyond N = 3; and the
    slowest-axis owner split gives every rank a contiguous range."""
    cc = umc.hypercubic_plaquettes(2)
    owner = umc.slowest_axis_owner(cc, 2)
    assert np.bincount(owner).tolist() == [32, 32]
    t = (np.arange(cc.sites()) % 16) // 8
    np.testing.assert_array_equal(owner, t)

    def create(**kw):
        d = umc.GaugeSlabDesc()
        d.model, d.N, d.cells, d.owner = umc.MODEL_SU, 3, cc._h, owner.ctypes.data_as(umc._vp)
        d.rank, d.world, d.coupling, d.width, d.hits, d.seed = 0, 2, 5.7, 0.3, 1, 1
        for k, v in kw.items():
            setattr(d, k, v)
        h = umc._vp()
        rc = umc.lib.umc_gslab_create(ctypes.byref(d), ctypes.byref(h))
        if rc == umc.OK:
            umc.lib.umc_gslab_destroy(h)
        return rc

    assert create(cells=None) == umc.ERR_INVALID_ARGUMENT
    assert create(owner=None) == umc.ERR_INVALID_ARGUMENT
    assert create(rank=2) == umc.ERR_INVALID_ARGUMENT
    assert create(world=0, rank=0) == umc.ERR_INVALID_ARGUMENT
    assert create(hits=0) == umc.ERR_INVALID_ARGUMENT
    assert create(coupling=float("nan")) == umc.ERR_INVALID_ARGUMENT
    assert create(N=4) == umc.ERR_UNSUPPORTED
    assert create(model=umc.MODEL_ISING) == umc.ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        umc.slowest_axis_owner(umc.CellComplex(5, [[0, 1, 2, 3]]), 2)


def test_slab_wolff_boundary_merge(umc):
    """The host merge of the slab Wolff flip (umc_slab_wolff_merge, no GPU):
    every rank joins the boundary labels along the activated bonds from each
    rank's last plane into the next rank's first plane (periodic), finds the
    seed's component, and keeps its own labels in it."""
    P, world = 4, 2
    first = np.array([[100, 101, 102, 103], [200, 201, 202, 203]], np.uint32)
    last = np.array([[110, 110, 112, 113], [210, 211, 212, 213]], np.uint32)
    up = np.array([[1, 0, 0, 1], [0, 1, 0, 0]], np.uint8)  # 110-200, 113-203, 211-101

    def merge(seed_root, rank, rank_seed_root=0xFFFFFFFF):
        out = np.zeros(2 * P + 1, np.uint32)
        n = umc._u32(0)
        rc = umc.lib.umc_slab_wolff_merge(world, P, umc._ptr(first.ravel()), umc._ptr(last.ravel()),
                                          umc._ptr(up.ravel()), seed_root, rank, umc._ptr(first[rank]),
                                          umc._ptr(last[rank]), rank_seed_root, umc._ptr(out), ctypes.byref(n))
        assert rc == umc.OK
        return out[: n.value].tolist()

    assert merge(200, 0) == [110] and merge(200, 1, 200) == [200]
    assert merge(203, 0) == [113] and merge(203, 1, 203) == [203]
    assert merge(101, 0) == [101] and merge(101, 1) == [211]
    # a seed whose cluster touches no boundary: only its own rank flips it
    assert merge(999, 0, 999) == [999] and merge(999, 1) == []
    # labels on both boundaries of one rank (110 is in its last plane twice)
    assert merge(110, 0, 110) == [110] and merge(110, 1) == [200]
    bad = umc.lib.umc_slab_wolff_merge(world, P, None, None, None, 0, 0, None, None, 0, None, None)
    assert bad == umc.ERR_INVALID_ARGUMENT
