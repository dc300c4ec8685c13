"""Failure detection without a GPU fault: a bounded device wait that runs out
(a barrier nothing completes) comes back as UMC_ERR_DEVICE_TIMEOUT with the
status bit set, and the same process keeps running chains afterwards."""
import numpy as np
import pytest

from helpers import square_edges

pytestmark = pytest.mark.gpu


def test_grid_barrier_timeout_is_reported_and_the_context_survives(umc, oracle):
    code, bits = umc.selftest_barrier_timeout(0)
    assert code == umc.ERR_DEVICE_TIMEOUT
    assert bits & 8
    assert "grid barrier" in umc._last_error().decode()
    # the context is usable: a bit-exact Ising chain right after
    L = 32
    g = umc.square_lattice(L, L)
    ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP, seed=3)
    rec = ch.metropolis(0.44, 5)
    assert np.all(np.isfinite(rec[:, 0]))
    code2, bits2 = umc.selftest_barrier_timeout(0)
    assert code2 == umc.ERR_DEVICE_TIMEOUT and bits2 & 8
