"""One lattice split into slabs over ranks (umc_slab_*, SlabChain): the ranks
together must run exactly the single-GPU chain of the same seed -- every site
draws from the keys of its global colour-major index and sums its neighbours
in the single-GPU kernels' order.  Ising is compared bit for bit, VectorSpin<3>
to the last bit where the FP32 arithmetic is the same (asserted exactly here).

Several ranks run here as processes on one GPU with the gloo backend: their
kernels never wait on one another (the halo exchange is a host-side
send/recv between passes), so this exercises the decomposition and its
exchanges without more GPUs."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _start(umc, model, dims, seed, s0):
    n = int(np.prod(dims))
    g = umc.cubic_lattice(*dims) if len(dims) == 3 and dims[2] > 1 else umc.square_lattice(dims[0], dims[1])
    if model == "ising":
        ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP, wolff_axis=umc.AXIS_FIXED,
                       seed=seed)
    else:
        ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE,
                       wolff_axis=umc.AXIS_SPHERE, seed=seed)
    ch.set_field(s0)
    return ch, n


def _initial(model, n, seed):
    rng = np.random.default_rng(seed)
    if model == "ising":
        return np.where(rng.random(n) < 0.5, -1, 1).astype(np.int8)
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _slab(umc, model, dims, rank, world, seed, group=None):
    if model == "ising":
        return umc.SlabChain(umc.MODEL_ISING, dims, rank=rank, world=world, group=group, coupling=1, seed=seed)
    return umc.SlabChain(umc.MODEL_VECTOR, dims, rank=rank, world=world, group=group, components=3, coupling=1.0,
                         proposal=umc.PROPOSAL_SPHERE, seed=seed)


@pytest.mark.parametrize("model,dims,beta", [("ising", (64, 32, 1), 0.44), ("ising", (8, 8, 8), 0.22),
                                              ("o3", (8, 8, 8), 0.693), ("o3", (16, 6, 1), 1.1)])
def test_single_slab_is_the_chain(umc, model, dims, beta):
    """world 1: the slab's halos are its own periodic planes."""
    ch, n = _start(umc, model, dims, 7, _initial(model, int(np.prod(dims)), 3))
    s0 = ch.get_field()
    rec_c = ch.metropolis(beta, 12)
    sl = _slab(umc, model, dims, 0, 1, 7)
    sl.set_field(s0)
    rec_s = sl.metropolis(beta, 12)
    np.testing.assert_array_equal(sl.gather_field().reshape(ch.get_field().shape), ch.get_field())
    np.testing.assert_allclose(rec_s[:, [0, 1, 7]], rec_c[:, [0, 1, 7]], rtol=1e-9, atol=1e-9)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, model, dims, beta, sweeps, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    import universal_classical_montecarlo_b200 as umc

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        n = int(np.prod(dims))
        s0 = _initial(model, n, 5)
        sl = _slab(umc, model, dims, rank, world, 11)
        sl.set_field(s0)
        rec = sl.metropolis(beta, sweeps)
        field = sl.gather_field()
        out[rank] = (field, rec, sl.planes_range)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("model,dims,world", [("ising", (32, 16, 1), 2), ("ising", (8, 8, 6), 3),
                                               ("o3", (8, 8, 8), 2), ("ising", (16, 2, 1), 2)])
def test_slabs_over_ranks_are_the_chain(umc, model, dims, world):
    """2 or 3 gloo ranks, one slab each (a rank may hold a single plane, whose
    two halos then come from different ranks -- or, with two ranks and two
    planes, both from the same one): the gathered lattice and the summed
    records equal the single-GPU chain's after 10 sweeps."""
    import torch.multiprocessing as mp

    beta = 0.44 if model == "ising" else 0.693
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), model, dims, beta, 10, out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    n = int(np.prod(dims))
    ch, _ = _start(umc, model, dims, 11, _initial(model, n, 5))
    rec_c = ch.metropolis(beta, 10)
    want = ch.get_field()
    ranges = [res[r][2] for r in range(world)]
    assert ranges[0][0] == 0 and all(ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))
    for r in range(world):
        field, rec, _ = res[r]
        np.testing.assert_array_equal(field.reshape(want.shape), want)
        np.testing.assert_allclose(rec[:, [0, 1, 7]], rec_c[:, [0, 1, 7]], rtol=1e-9, atol=1e-9)


def _program(obj, beta):
    """2 sweeps, 6 Wolff flips, 1 sweep: the cluster sizes and the records."""
    r1 = obj.metropolis(beta, 2)
    sizes = obj.wolff(beta, 6)
    if isinstance(sizes, tuple):  # Chain.wolff returns (sizes, records)
        sizes = sizes[0]
    r2 = obj.metropolis(beta, 1)
    return np.asarray(sizes, np.uint64), np.concatenate([r1, r2])


@pytest.mark.parametrize("model,dims,beta", [("ising", (32, 16, 1), 0.44), ("ising", (8, 8, 6), 0.25),
                                              ("o3", (8, 8, 8), 0.75), ("ising", (16, 2, 1), 0.6)])
def test_single_slab_wolff_is_the_chain(umc, model, dims, beta):
    """world 1: the last plane's bonds into the next plane close the periodic
    lattice through the slab's own halo and the host merge."""
    ch, n = _start(umc, model, dims, 7, _initial(model, int(np.prod(dims)), 3))
    s0 = ch.get_field()
    sizes_c, rec_c = _program(ch, beta)
    sl = _slab(umc, model, dims, 0, 1, 7)
    sl.set_field(s0)
    sizes_s, rec_s = _program(sl, beta)
    np.testing.assert_array_equal(sizes_s, sizes_c)
    assert sizes_c.max() > 1
    np.testing.assert_array_equal(sl.gather_field().reshape(ch.get_field().shape), ch.get_field())
    np.testing.assert_allclose(rec_s[:, [0, 1, 7]], rec_c[:, [0, 1, 7]], rtol=1e-9, atol=1e-9)


def _wolff_worker(rank, world, port, model, dims, beta, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    import universal_classical_montecarlo_b200 as umc

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        n = int(np.prod(dims))
        sl = _slab(umc, model, dims, rank, world, 11)
        sl.set_field(_initial(model, n, 5))
        sizes, rec = _program(sl, beta)
        out[rank] = (sl.gather_field(), sizes, rec)
        sl.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("model,dims,beta,world", [("ising", (32, 16, 1), 0.44, 2), ("ising", (8, 8, 6), 0.25, 3),
                                                    ("o3", (8, 8, 8), 0.75, 2), ("ising", (16, 2, 1), 0.6, 2)])
def test_slab_wolff_over_ranks_is_the_chain(umc, model, dims, beta, world):
    """Wolff flips whose clusters cross the slabs (a cross-rank merge of the
    boundary labels), between Metropolis sweeps: cluster sizes, the gathered
    lattice and the summed records equal the single-GPU chain's."""
    import torch.multiprocessing as mp

    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_wolff_worker, args=(world, _free_port(), model, dims, beta, out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    n = int(np.prod(dims))
    ch, _ = _start(umc, model, dims, 11, _initial(model, n, 5))
    sizes_c, rec_c = _program(ch, beta)
    assert sizes_c.max() > 1
    for r in range(world):
        field, sizes, rec = res[r]
        np.testing.assert_array_equal(sizes, sizes_c)
        np.testing.assert_array_equal(field.reshape(ch.get_field().shape), ch.get_field())
        np.testing.assert_allclose(rec[:, [0, 1, 7]], rec_c[:, [0, 1, 7]], rtol=1e-9, atol=1e-9)
