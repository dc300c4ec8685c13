"""The allocation-free Wolff entry point (umc_wolff_flip_noalloc).

It serves callers that cannot call cudaMalloc: they own the field and the graph
in device memory already, and the flip's scratch comes from a static device
array inside the library.  Here it must reproduce the chain entry point
(umc_wolff_run) exactly -- same kernels, same keyed random streams -- on two
consecutive flips, for Ising and for O(3).  This file is collected last so a
failure here never hides the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import cubic_edges, random_unit_vectors, relabel_edges, square_edges

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _entry(umc):
    f = umc.lib.umc_wolff_flip_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_double, C.c_double, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p]
    return f


def _device_csr(torch, oracle, g, ei, ej):
    """Colour-major CSR of an engine graph (the chain's own site order)."""
    _, _, pos = g.colouring()
    ri, rj = relabel_edges(ei, ej, pos)
    st, off, bonds, slot = oracle.pair_graph(g.sites(), ri, rj)
    assert st == 0
    dev = [torch.from_numpy(a.view(np.int32)).cuda() for a in (off, bonds, slot)]
    return pos, dev


def _run_noalloc(umc, torch, model, comps, field_dev, n, csr, J, beta, seed, flip):
    size = C.c_uint64(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = _entry(umc)(model, comps, field_dev.data_ptr(), n, csr[0].data_ptr(), csr[1].data_ptr(),
                     csr[2].data_ptr(), J, beta, seed, flip, C.byref(size), stream)
    umc.check(rc)
    return size.value


def test_noalloc_ising_matches_chain(umc, oracle):
    torch = pytest.importorskip("torch")
    L, beta, seed = 32, 0.44, 5
    g = umc.square_lattice(L, L)
    n = L * L
    pos, csr = _device_csr(torch, oracle, g, *square_edges(L, L))
    s0 = np.where(np.random.default_rng(1).random(n) < 0.5, -1, 1).astype(np.int8)
    cm = np.empty(n, np.int8)
    cm[pos] = s0
    field = torch.from_numpy(cm).cuda()
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP,
                   wolff_axis=umc.AXIS_FIXED, seed=seed)
    ch.set_field(s0)
    sizes_chain, _ = ch.wolff(beta, 2, records=False)
    sizes = [_run_noalloc(umc, torch, umc.MODEL_ISING, 1, field, n, csr, 1.0, beta, seed, f) for f in (0, 1)]
    assert sizes == [int(x) for x in sizes_chain]
    got = field.cpu().numpy()[pos]
    np.testing.assert_array_equal(got, ch.get_field())


def test_noalloc_o3_matches_chain(umc, oracle):
    torch = pytest.importorskip("torch")
    L, beta, seed = 8, 0.693, 9
    g = umc.cubic_lattice(L, L, L)
    n = L**3
    pos, csr = _device_csr(torch, oracle, g, *cubic_edges(L, L, L))
    v0 = random_unit_vectors(n, 3, 2).astype(np.float32)
    soa = np.empty((3, n), np.float32)
    soa[:, pos] = v0.T
    field = torch.from_numpy(soa.reshape(-1).copy()).cuda()
    ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE,
                   wolff_axis=umc.AXIS_SPHERE, seed=seed)
    ch.set_field(v0)
    sizes_chain, _ = ch.wolff(beta, 2, records=False)
    sizes = [_run_noalloc(umc, torch, umc.MODEL_VECTOR, 3, field, n, csr, 1.0, beta, seed, f) for f in (0, 1)]
    assert sizes == [int(x) for x in sizes_chain]
    got = field.cpu().numpy().reshape(3, n)[:, pos].T
    np.testing.assert_allclose(got, ch.get_field(), rtol=0, atol=TOL)


def test_noalloc_rejects_graphs_above_its_scratch(umc, oracle):
    torch = pytest.importorskip("torch")
    g = umc.square_lattice(4, 4)
    _, csr = _device_csr(torch, oracle, g, *square_edges(4, 4))
    field = torch.ones(16, dtype=torch.int8, device="cuda")
    size = C.c_uint64(0)
    rc = _entry(umc)(umc.MODEL_ISING, 1, field.data_ptr(), (1 << 20) + 1, csr[0].data_ptr(), csr[1].data_ptr(),
                     csr[2].data_ptr(), 1.0, 0.4, 1, 0, C.byref(size), torch.cuda.current_stream().cuda_stream)
    assert rc == umc.ERR_UNSUPPORTED
    assert "1,048,576" in umc.lib.umc_last_error().decode()


def test_noalloc_refuses_a_bad_csr_and_stays_usable(umc, oracle):
    """A neighbour id beyond the graph, a self-loop and a bond stored at one
    end only are refused by the device check before any flip kernel runs;
    the field is untouched and the next valid call flips as the chain does."""
    torch = pytest.importorskip("torch")
    L, beta, seed = 8, 0.44, 3
    g = umc.square_lattice(L, L)
    n = L * L
    pos, csr = _device_csr(torch, oracle, g, *square_edges(L, L))
    off = csr[0].cpu().numpy().view(np.uint32)
    bonds = csr[1].cpu().numpy().view(np.uint32)
    field = torch.ones(n, dtype=torch.int8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def call(b):
        size = C.c_uint64(0)
        dev = torch.from_numpy(b.view(np.int32)).cuda()
        rc = _entry(umc)(umc.MODEL_ISING, 1, field.data_ptr(), n, csr[0].data_ptr(), dev.data_ptr(),
                         csr[2].data_ptr(), 1.0, beta, seed, 0, C.byref(size), stream)
        return rc, umc.lib.umc_last_error().decode()

    out_of_range = bonds.copy()
    out_of_range[5] = n + 7  # in-bounds slot, id beyond the graph
    self_loop = bonds.copy()
    self_loop[off[9]] = 9
    one_sided = bonds.copy()
    i, j = 10, int(bonds[off[10]])
    one_sided[off[10]] = int(bonds[off[10] + 1])  # row 10 loses its bond to j, j keeps its bond to 10
    for bad, words in ((out_of_range, "neighbour id"), (self_loop, "self-loop"), (one_sided, "not symmetric")):
        rc, msg = call(bad)
        assert rc == umc.ERR_INVALID_ARGUMENT and words in msg, (rc, msg)
        assert bool((field == 1).all()), "a refused call changed the field"
    rc, msg = call(bonds.copy())
    assert rc == umc.OK, msg
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP, wolff_axis=umc.AXIS_FIXED,
                   seed=seed)
    ch.set_field(np.ones(n, np.int8))
    ch.wolff(beta, 1, records=False)
    np.testing.assert_array_equal(field.cpu().numpy()[pos], ch.get_field())
