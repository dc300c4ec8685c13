"""One gauge lattice split over ranks (umc_gslab_*, GaugeSlab): the ranks
together must run exactly the single-GPU chain of the same seed -- each link
draws from the keys of its global colour-major index and sums its plaquettes
in the single-GPU order, so SU(N) (FP32 decisions) and U(1) links agree bit
for bit, and the summed records agree to FP64 summation order.

Several ranks run here as processes on one GPU with the gloo backend: their
kernels never wait on one another (the links of each colour class move
host-side between passes), so this exercises the decomposition and its
exchanges without more GPUs."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# name: (model, N, cells builder and size, beta, width, hits)
CASES = {
    "su3_4d": ("su", 3, ("hypercubic", 4), 5.7, 0.3, 2),
    "su2_4d": ("su", 2, ("hypercubic", 4), 2.3, 0.4, 1),
    "u1_4d": ("u1", 1, ("hypercubic", 4), 1.0, 0.7, 2),
    "u1_2d": ("u1", 1, ("square", 12), 2.0, 0.9, 1),
}


def _cells(umc, spec):
    kind, L = spec
    return umc.hypercubic_plaquettes(L) if kind == "hypercubic" else umc.square_plaquettes(L)


def _chain(umc, case, seed):
    model, N, spec, beta, width, hits = CASES[case]
    cc = _cells(umc, spec)
    if model == "su":
        ch = umc.Chain(umc.MODEL_SU, cells=cc, components=N, coupling=beta, proposal=umc.PROPOSAL_SUSHIFT,
                       width=width, hits=hits, seed=seed)
    else:
        ch = umc.Chain(umc.MODEL_U1, cells=cc, coupling=beta, proposal=umc.PROPOSAL_U1SHIFT, width=width, hits=hits,
                       seed=seed)
    return ch, cc


def _slab(umc, case, cc, rank, world, seed, group=None):
    model, N, spec, beta, width, hits = CASES[case]
    owner = umc.slowest_axis_owner(cc, world)
    m = umc.MODEL_SU if model == "su" else umc.MODEL_U1
    return umc.GaugeSlab(m, cc, owner, rank=rank, world=world, group=group, N=N, coupling=beta, width=width,
                         hits=hits, seed=seed)


def _start_field(umc, case):
    """A hot start from the single-GPU chain's own randomisation."""
    ch, cc = _chain(umc, case, 1)
    ch.randomize(5)
    return ch.get_field().reshape(cc.sites(), -1).copy()


@pytest.mark.parametrize("case", list(CASES))
def test_single_gauge_slab_is_the_chain(umc, case):
    """world 1: every link owned, no halo."""
    s0 = _start_field(umc, case)
    ch, cc = _chain(umc, case, 7)
    ch.set_field(s0)
    rec_c = ch.metropolis(1.0, 3)
    sl = _slab(umc, case, cc, 0, 1, 7)
    assert sl.n_owned == sl.n_local == cc.sites()
    sl.set_field(s0)
    rec_s = sl.metropolis(1.0, 3)
    np.testing.assert_array_equal(sl.gather_field(), ch.get_field().reshape(cc.sites(), -1))
    np.testing.assert_allclose(rec_s[:, [0, 1, 2, 7]], rec_c[:, [0, 1, 2, 7]], rtol=1e-9, atol=1e-9)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, s0, sweeps, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    import universal_classical_montecarlo_b200 as umc

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        cc = _cells(umc, CASES[case][2])
        sl = _slab(umc, case, cc, rank, world, 11)
        sl.set_field(s0)
        rec = sl.metropolis(1.0, sweeps)
        field = sl.gather_field()
        out[rank] = (field, rec, sl.n_owned, sl.n_local, len(sl.counts))
        sl.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,world", [("su3_4d", 2), ("su3_4d", 3), ("u1_4d", 3), ("u1_2d", 4), ("su2_4d", 2)])
def test_gauge_slabs_over_ranks_are_the_chain(umc, case, world):
    """2 to 4 gloo ranks, a range of the slowest coordinate each (with L = 4 and
    3 ranks, ranks of a single slice whose two halo slices come from
    different ranks): the gathered links and the summed records equal the
    single-GPU chain's after 3 sweeps."""
    import torch.multiprocessing as mp

    s0 = _start_field(umc, case)
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), case, s0, 3, out), nprocs=world, start_method="spawn",
                           join=True)
        res = dict(out)
    ch, cc = _chain(umc, case, 11)
    ch.set_field(s0)
    rec_c = ch.metropolis(1.0, 3)
    want = ch.get_field().reshape(cc.sites(), -1)
    assert sum(res[r][2] for r in range(world)) == cc.sites()
    for r in range(world):
        field, rec, n_owned, n_local, peers = res[r]
        assert n_local > n_owned and peers > 0  # a real halo, exchanged
        np.testing.assert_array_equal(field, want)
        np.testing.assert_allclose(rec[:, [0, 1, 2, 7]], rec_c[:, [0, 1, 2, 7]], rtol=1e-9, atol=1e-9)
