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
    with mp.Manager() as mgr:
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
