"""Chain checkpoints (umc_chain_checkpoint / umc_chain_restore): a chain
restored from an image taken mid-run -- into a fresh chain created with
another seed, or through a file -- continues bit for bit as the original, for
spin and gauge models; images of another model, size or coupling, and damaged
images, are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _make(umc, kind, seed):
    if kind == "o3":
        return umc.Chain(umc.MODEL_VECTOR, graph=umc.cubic_lattice(8, 8, 8), components=3, coupling=1.0,
                         proposal=umc.PROPOSAL_SPHERE, wolff_axis=umc.AXIS_SPHERE, seed=seed)
    if kind == "ising":
        return umc.Chain(umc.MODEL_ISING, graph=umc.square_lattice(32, 32), coupling=1, proposal=umc.PROPOSAL_FLIP,
                         wolff_axis=umc.AXIS_FIXED, seed=seed)
    return umc.Chain(umc.MODEL_SU, cells=umc.hypercubic_plaquettes(4), components=2, coupling=2.3,
                     proposal=umc.PROPOSAL_SUSHIFT, width=0.3, hits=2, seed=seed)


def _advance(ch, kind, n):
    if kind == "su2":
        return ch.metropolis(1.0, n), None
    sizes, rec = ch.hybrid(0.693 if kind == "o3" else 0.44, n)
    return rec, sizes


@pytest.mark.parametrize("kind", ["o3", "ising", "su2"])
def test_restored_chain_continues_exactly(umc, kind, tmp_path):
    a = _make(umc, kind, 11)
    a.randomize(3)
    _advance(a, kind, 6)
    image = a.checkpoint()
    a.save(tmp_path / "chain.ckpt")
    ra, sa = _advance(a, kind, 8)
    fa = a.get_field()
    stats_a = a.wolff_stats()
    for via_file in (False, True):
        b = _make(umc, kind, 999)  # another seed: the image carries the key seed
        if via_file:
            b.load(tmp_path / "chain.ckpt")
        else:
            b.restore(image)
        assert b.counters() == (6, 6) if kind != "su2" else b.counters()[0] == 6
        rb, sb = _advance(b, kind, 8)
        np.testing.assert_array_equal(ra, rb)
        if sa is not None:
            np.testing.assert_array_equal(sa, sb)
        np.testing.assert_array_equal(fa, b.get_field())
        # the image carries the Wolff statistics behind mean_cluster_size
        assert b.wolff_stats() == stats_a


def test_version1_image_is_accepted_and_restarts_the_wolff_statistics(umc):
    """An image in the earlier 88-byte-header layout (no Wolff statistics)
    still restores the field, seed and counters; mean_cluster_size then counts
    only the flips made after the restore."""
    a = _make(umc, "o3", 11)
    a.randomize(3)
    _advance(a, "o3", 6)
    v2 = bytearray(a.checkpoint())
    assert int.from_bytes(v2[8:12], "little") == 2
    v1 = bytearray(v2[:88] + v2[104:])
    v1[8:12] = (1).to_bytes(4, "little")
    ra, sa = _advance(a, "o3", 5)
    b = _make(umc, "o3", 999)
    b.restore(bytes(v1))
    assert b.counters() == (6, 6) and b.wolff_stats() == (0, 0.0)
    rb, sb = _advance(b, "o3", 5)
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(sa, sb)
    assert b.wolff_stats() == (5, float(np.sum(sb)))


def test_mismatched_or_damaged_images_are_refused(umc):
    a = _make(umc, "o3", 1)
    image = a.checkpoint()
    other_size = umc.Chain(umc.MODEL_VECTOR, graph=umc.cubic_lattice(8, 8, 4), components=3, coupling=1.0,
                           proposal=umc.PROPOSAL_SPHERE, wolff_axis=umc.AXIS_SPHERE, seed=1)
    other_coupling = umc.Chain(umc.MODEL_VECTOR, graph=umc.cubic_lattice(8, 8, 8), components=3, coupling=0.5,
                               proposal=umc.PROPOSAL_SPHERE, wolff_axis=umc.AXIS_SPHERE, seed=1)
    ising = _make(umc, "ising", 1)
    for ch in (other_size, other_coupling, ising):
        with pytest.raises(ValueError):
            ch.restore(image)
    damaged = bytearray(image)
    damaged[0] ^= 0xFF
    with pytest.raises(ValueError):
        a.restore(bytes(damaged))
    with pytest.raises(ValueError):
        a.restore(image[:-4])
    # the refused restores left the chain as it was
    np.testing.assert_array_equal(np.frombuffer(a.checkpoint(), np.uint8), np.frombuffer(image, np.uint8))


def test_learned_batch_and_network_continue_exactly(umc, tmp_path):
    """The C5 state -- the batch's angles and sweep counter, and the network --
    saved mid-run and loaded into fresh objects continues the learned sweeps
    bit for bit."""
    a = umc.U1Batch(8, 16, 3.0, width=0.5, seed=4)
    a.run(30, records=False)
    net = umc.ProposalNet(5)
    a.save(tmp_path / "batch.npz")
    net.save(tmp_path / "net.npy")
    ra = a.run(10, net)
    b = umc.U1Batch(8, 16, 3.0, width=0.5, seed=4)
    b.load(tmp_path / "batch.npz")
    net2 = umc.ProposalNet(77)
    net2.load(tmp_path / "net.npy")
    rb = b.run(10, net2)
    np.testing.assert_array_equal(ra, rb)
    for c in range(8):
        np.testing.assert_array_equal(a.get_field(c), b.get_field(c))
    other = umc.U1Batch(8, 16, 3.0, width=0.5, seed=5)
    with pytest.raises(ValueError):
        other.load(tmp_path / "batch.npz")


def test_replica_exchange_batch_continues_exactly(umc, tmp_path):
    """Fields, counters and the temperature map saved after some exchange
    rounds and loaded into a fresh batch continue the ladders exactly; a
    holder that is not a permutation of a ladder's chains is refused."""
    Ls = np.array([16, 32])
    betas = np.stack([np.geomspace(0.8, 1.3, 4)] * 2)
    a = umc.Batch(Ls, betas, width=1.0, sweeps_per_exchange=3, seed=9)
    a.randomize(2)
    a.run(5)
    a.save(tmp_path / "ladders.npz")
    ra = a.run(4)
    b = umc.Batch(Ls, betas, width=1.0, sweeps_per_exchange=3, seed=9)
    b.load(tmp_path / "ladders.npz")
    rb = b.run(4)
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(a.temperature_map(), b.temperature_map())
    assert a.counters() == b.counters()
    for c in range(a.n_chains):
        np.testing.assert_array_equal(a.get_field(c), b.get_field(c))
    bad = np.arange(8, dtype=np.uint32)[::-1].copy()  # swaps chains across ladders
    with pytest.raises(ValueError):
        umc.check(umc.lib.umc_batch_set_state(b._h, 0, 0, 0, bad.ctypes.data_as(umc._vp)))
