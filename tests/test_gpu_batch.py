"""Batched XY chains with replica-exchange ladders (umc_batch_*), through the C ABI.

Every chain is checked segment by segment against the single-chain oracle
(the reference's PairModel / U1Shift arithmetic on a checkerboard-relabelled
square lattice, keyed by the chain's seed) and the exchange round against the
oracle's swap rule, both from identical states.
"""
import os

import numpy as np
import pytest

from helpers import checker_position, relabel_edges, square_edges

HERE = os.path.dirname(os.path.abspath(__file__))

pytestmark = pytest.mark.gpu

TOL = 4e-5     # radians after one segment (10 sweeps)
# the kernel decides as the FP64 test does on its FP32 angles; only the FP32
# rounding of the proposed angle (about 2.4e-7, moving log_p by < 1.5e-6 at
# beta <= 1.3) separates its decisions from the oracle's
MARGIN = 2e-5


def _geometric(lo, hi, R):
    return lo * (hi / lo) ** (np.arange(R) / max(1, R - 1))


def test_batch_segments_match_oracle(umc, oracle):
    Ls = [8, 16, 12]
    R, S = 4, 3
    betas = np.stack([_geometric(0.8, 1.3, R)] * len(Ls))
    b = umc.Batch(Ls, betas, coupling=1.0, width=1.0, sweeps_per_exchange=S, seed=7)
    b.randomize(3)
    cseeds, lseeds = b.seeds()
    csr = {}
    for L in set(Ls):
        pos = checker_position(L, L)
        ei, ej = relabel_edges(*square_edges(L, L), pos)
        st, off, bonds, _ = oracle.pair_graph(L * L, ei, ej)
        csr[L] = (pos, off, bonds)
    for seg in range(3):
        holder = b.temperature_map()
        fields = [b.get_field(c).astype(np.float64) for c in range(b.n_chains)]
        energies = np.zeros(b.n_chains)
        expect = []
        near = False
        for c in range(b.n_chains):
            l, L = c // R, b.chain_side(c)
            slot = int(np.nonzero(holder[l] == c)[0][0])
            pos, off, bonds = csr[L]
            cm = np.empty(L * L)
            cm[pos] = fields[c]
            t_o, obs, margin = oracle.xy_metropolis(off, bonds, 1.0, betas[l, slot], 1.0, int(cseeds[c]), seg * S, S, cm)
            near |= bool((np.abs(margin) < MARGIN).any())
            energies[c] = obs[-1, 0]
            expect.append(t_o[pos])
        rec = b.run(1)
        for c in range(b.n_chains):
            got = b.get_field(c).astype(np.float64)
            d = np.abs(np.angle(np.exp(1j * (got - expect[c]))))
            if not near:
                assert d.max() < TOL, (seg, c, d.max())
        # exchange round: the oracle's rule on the oracle energies
        new_holder = b.temperature_map()
        for l in range(len(Ls)):
            h_o, acc = oracle.replica_exchange(betas[l], holder[l], energies, int(lseeds[l]), seg, seg & 1)
            np.testing.assert_array_equal(new_holder[l], h_o)
        # records: slot k's energy is the energy of its holder before the exchange
        for l in range(len(Ls)):
            for k in range(R):
                c = int(rec[0, l, k, 3])
                assert c == holder[l, k]
                assert abs(rec[0, l, k, 0] - energies[c]) < 1e-3 * max(1, abs(energies[c]))
    s, r, w = b.counters()
    assert (s, r) == (3 * S, 3)


def test_batch_is_deterministic_and_config_independent(umc):
    Ls = [16, 32, 64, 128, 256, 32]
    R = 8
    betas = np.stack([_geometric(0.8, 1.3, R)] * len(Ls))
    a = umc.Batch(Ls, betas, seed=11)
    b = umc.Batch(Ls, betas, seed=11)
    for x in (a, b):
        x.randomize(5)
    ra, rb = a.run(6), b.run(6)
    np.testing.assert_array_equal(ra, rb)
    for c in (0, R * 4, a.n_chains - 1):
        np.testing.assert_array_equal(a.get_field(c), b.get_field(c))
    sw = a.counters()
    assert sw[0] == 60 and sw[1] == 6 and sw[2] > 0
    assert np.isfinite(ra).all()
    # every temperature slot is held by exactly one chain of its ladder
    h = a.temperature_map()
    for l in range(len(Ls)):
        assert sorted(h[l]) == list(range(l * R, (l + 1) * R))
    assert a.config(256)["block"] in (256, 512, 1024)


def test_batch_energy_per_site_orders_with_beta(umc):
    # hotter slots carry higher energy on average (a sanity check of the ladder)
    R = 8
    betas = np.stack([_geometric(0.5, 1.5, R)] * 2)
    b = umc.Batch([32, 32], betas, seed=3)
    b.randomize(1)
    b.run(20)
    rec = b.run(40)
    e = rec[:, :, :, 0].mean(axis=0) / (32 * 32)
    assert (np.diff(e, axis=1) < 0.02).all()
    assert e[0, 0] > e[0, -1]


def test_autotuner_file_cache(tmp_path):
    """With UMC_TUNE_CACHE set, a batch's tuned launch shapes are appended to
    that file keyed by (GPU, kernel, L, chains, sweeps per exchange), and a
    later process takes them from the file instead of timing candidates: an
    entry edited by hand is what the next batch uses."""
    import subprocess
    import sys

    root = os.path.dirname(HERE)
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import numpy as np, universal_classical_montecarlo_b200 as umc\n"
            "b = umc.Batch([16, 32], np.stack([np.geomspace(0.8, 1.3, 4)] * 2), width=1.0, sweeps_per_exchange=3)\n"
            "print(*[b.config(L)[k] for L in (16, 32) for k in ('chains_per_cta', 'ctas_per_chain', 'block')])\n"
            ) % root
    path = tmp_path / "tune.txt"
    env = dict(os.environ, UMC_TUNE_CACHE=str(path))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    text = path.read_text()
    seg = [ln for ln in text.splitlines() if "/xy_batch_segment/" in ln]
    assert len(seg) == 2 and any("/L16/" in ln for ln in seg) and any("/L32/" in ln for ln in seg)
    assert sum("/xy_batch_persistent/" in ln for ln in text.splitlines()) == 1
    first = [int(v) for v in r.stdout.split()]
    # hand-edit the L = 16 entry: one chain per CTA, 64 threads
    text = "\n".join(ln if "/xy_batch_segment/L16/" not in ln else ln.split()[0] + " 1 1 64"
                     for ln in path.read_text().splitlines())
    path.write_text(text + "\n")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    second = [int(v) for v in r.stdout.split()]
    assert second[:3] == [1, 1, 64] and second[3:] == first[3:]
    assert len(path.read_text().split()) == 12  # nothing re-tuned, nothing appended


def test_sharded_batch_equals_the_whole_batch(umc):
    """The ladders shard over ranks with no exchange between shards: the two
    shards of a 2-rank split (run here one after the other on one GPU, no
    kernel waiting on another) reproduce the unsharded batch -- the same
    chain and ladder keys, fields bit for bit, the same temperature maps and
    records (energies to FP64 summation order)."""
    Ls = np.array([16, 32, 16, 8, 32])
    R = 4
    betas = np.stack([_geometric(0.8, 1.3, R)] * len(Ls))
    whole = umc.Batch(Ls, betas, width=1.0, sweeps_per_exchange=3, seed=21)
    whole.randomize(8)
    rec_w = whole.run(4)
    parts, recs = [], []
    for rank in range(2):
        b = umc.Batch.shard(Ls, betas, rank, 2, width=1.0, sweeps_per_exchange=3, seed=21)
        b.randomize(8)
        recs.append(b.run(4))
        parts.append(b)
    lo1 = parts[1].ladder_range[0]
    assert parts[0].ladder_range == (0, lo1) and parts[1].ladder_range == (lo1, len(Ls))
    cs_w, ls_w = whole.seeds()
    cs = np.concatenate([p.seeds()[0] for p in parts])
    ls = np.concatenate([p.seeds()[1] for p in parts])
    np.testing.assert_array_equal(cs, cs_w)
    np.testing.assert_array_equal(ls, ls_w)
    recs[1][..., 3] += lo1 * R  # a shard's records name its chains by local index
    rec = np.concatenate(recs, axis=1)
    np.testing.assert_array_equal(rec[..., 3], rec_w[..., 3])  # which chain held each slot
    np.testing.assert_allclose(rec, rec_w, rtol=1e-12, atol=1e-9)
    tmap = np.concatenate([p.temperature_map() + p.ladder_range[0] * R for p in parts])
    np.testing.assert_array_equal(tmap, whole.temperature_map())
    for c in range(whole.n_chains):
        p = parts[0] if c < lo1 * R else parts[1]
        np.testing.assert_array_equal(p.get_field(c - p.ladder_range[0] * R), whole.get_field(c))


def test_sharded_u1batch_equals_the_whole_batch(umc):
    whole = umc.U1Batch(7, 8, 2.0, width=0.5, seed=3)
    whole.randomize(4)
    rec_w = whole.run(5)
    recs, parts = [], []
    for rank in range(3):
        b = umc.U1Batch.shard(7, 8, 2.0, rank, 3, width=0.5, seed=3)
        b.randomize(4)
        recs.append(b.run(5))
        parts.append(b)
    np.testing.assert_array_equal(np.concatenate([p.seeds() for p in parts]), whole.seeds())
    np.testing.assert_allclose(np.concatenate(recs, axis=1), rec_w, rtol=1e-12, atol=1e-12)
    c = 0
    for p in parts:
        for k in range(p.n_chains):
            np.testing.assert_array_equal(p.get_field(k), whole.get_field(c))
            c += 1


@pytest.mark.parametrize("cluster,ctas_per_sm", [(1, 1), (1, 2), (4, 1), (4, 2), (8, 1), (8, 2)])
def test_persistent_segment_equals_grouped_segments(umc, cluster, ctas_per_sm):
    """The one-kernel segment (resident CTAs taking work items, a 256^2 chain
    swept by one CTA or a cluster of CTAs, small chains packed, the exchanges
    run by whichever CTA completes a ladder) and the per-group kernels run
    the same chains and exchanges: fields bit for bit, temperature maps and
    records equal (energies to FP64 summation order), and both advance the
    counters by every segment.  Creation selects the form that measured
    faster; every persistent variant is forced here."""
    Ls = np.array([256, 16, 64, 32, 256, 128, 16])
    R, S, n = 4, 4, 5
    betas = np.stack([_geometric(0.8, 1.3, R)] * len(Ls))
    a = umc.Batch(Ls, betas, width=1.0, sweeps_per_exchange=S, seed=5)
    b = umc.Batch(Ls, betas, width=1.0, sweeps_per_exchange=S, seed=5)
    a.set_persistent_config(cluster, ctas_per_sm)
    b.set_persistent(False)
    info = a.persistent_info()
    assert info["enabled"] and info["grid"] % info["cluster"] == 0
    assert (info["cluster"], info["ctas_per_sm"]) == (cluster, ctas_per_sm)
    assert info["big_items"] == 2 * R
    assert not b.persistent_info()["enabled"]
    for x in (a, b):
        x.randomize(6)
    ra, rb = a.run(n), b.run(n)
    assert a.counters()[:2] == (n * S, n)
    np.testing.assert_array_equal(ra[..., 3], rb[..., 3])
    np.testing.assert_allclose(ra, rb, rtol=1e-12, atol=1e-9)
    np.testing.assert_array_equal(a.temperature_map(), b.temperature_map())
    assert a.counters() == b.counters()
    for c in range(a.n_chains):
        np.testing.assert_array_equal(a.get_field(c), b.get_field(c))
    assert a.sites()[1] == n  # one kernel per segment


def _check_wrapped(got, th):
    far = np.abs(th) > 8
    np.testing.assert_array_equal(got[~far], th[~far])
    assert np.all(np.abs(got[far]) <= np.pi + 1e-6)
    d = np.angle(np.exp(1j * (got[far].astype(np.float64) - th[far].astype(np.float64))))
    np.testing.assert_allclose(d, 0, atol=1e-6)


def test_uploaded_angles_outside_the_sincos_domain_are_wrapped(umc):
    """The FP32 XY decisions bound __sincosf's error for |angle| <= 8; an
    uploaded angle beyond that is stored as the same angle in [-pi, pi], and
    every other angle exactly as given (batched and single chains)."""
    L = 8
    th = np.random.default_rng(0).uniform(-7.9, 7.9, L * L).astype(np.float32)
    th[:6] = np.float32([100.0, -50.5, 8.5, -8.0001, 1e6, 8.0])
    b = umc.Batch([L], np.array([[1.0, 1.1]]), width=1.0, seed=2)
    b.set_field(0, th)
    _check_wrapped(b.get_field(0), th)
    ch = umc.Chain(umc.MODEL_XY_ANGLE, graph=umc.square_lattice(L, L), coupling=1.0,
                   proposal=umc.PROPOSAL_U1SHIFT, width=1.0, seed=4)
    ch.set_field(th)
    _check_wrapped(ch.get_field(), th)
    ch.upload_async(th)
    _check_wrapped(ch.get_field(), th)
