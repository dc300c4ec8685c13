"""The N > 1 host path of bench.py with world_size 2 on CPU (gloo): every rank
runs its own replica chain, and the line reports the slowest rank's device
time and the units of all ranks.  No GPU is involved."""
import importlib.util
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    bench = _bench()
    ws, r, local = bench.rank_info()
    ms, units, e2e = bench.aggregate_ranks(dist, torch, "cpu", 10.0 + rank, 1000.0 * (rank + 1), 5.0 * (rank + 1))
    ms2, units2, none = bench.aggregate_ranks(dist, torch, "cpu", 1.0, 2.0, None)
    out[rank] = (ws, r, local, ms, units, e2e, ms2, units2, none)
    dist.destroy_process_group()


def test_replicas_aggregate_over_two_gloo_ranks():
    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    for rank in range(world):
        ws, r, local, ms, units, e2e, ms2, units2, none = res[rank]
        assert (ws, r, local) == (2, rank, rank)
        assert ms == 11.0  # the slowest rank
        assert units == 3000.0  # every rank's work
        assert e2e == 15.0
        assert (ms2, units2, none) == (1.0, 4.0, None)


def test_single_rank_defaults(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert _bench().rank_info() == (1, 0, 0)


# ----------------------------------- sharded batches (ladders or chains over ranks)
def test_shard_ranges_partition_the_units():
    import universal_classical_montecarlo_b200 as umc

    for n in (0, 1, 5, 32, 444):
        for world in (1, 2, 3, 8):
            ranges = [umc.shard_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))
            sizes = [hi - lo for lo, hi in ranges]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        umc.shard_range(4, 2, 2)


def _gather_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import numpy as np

    import universal_classical_montecarlo_b200 as umc

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    # records of a 7-ladder batch, ladders sharded over the ranks: (segments, ladders, replicas, 4)
    full = np.arange(3 * 7 * 4 * 4, dtype=np.float64).reshape(3, 7, 4, 4)
    lo, hi = umc.shard_range(7, rank, world)
    out[rank] = umc.gather_shards(full[:, lo:hi])
    dist.destroy_process_group()


def test_sharded_records_gather_in_rank_order_over_two_gloo_ranks():
    """Each rank holds the records of its ladders; gather_shards puts every
    rank's shard back in ladder order on every rank, as one unsharded batch's
    records."""
    import numpy as np

    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_gather_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn",
                           join=True)
        res = dict(out)
    full = np.arange(3 * 7 * 4 * 4, dtype=np.float64).reshape(3, 7, 4, 4)
    for rank in range(world):
        np.testing.assert_array_equal(res[rank], full)
