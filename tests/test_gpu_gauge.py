"""GPU parity for the gauge models (U(1) angles, SU(2)/SU(3) links) through the C ABI.

Each sweep starts from an identical state on both sides: the double-precision
oracle (CellModel + U1PlaquetteTerm / SUPlaquetteTerm arithmetic, multi-hit in
link order) and the engine (staple per link, FP32, SU(N) reunitarised).  Links
must agree within TOL except where the oracle's accept decision sat within
MARGIN of its threshold (and the links that share a cell with those).

For U(1) the engine decides as the FP64 test does on its FP32 links (FP32
first, FP64 inside the FP32 error band), so MARGIN_U1 only covers the FP32
rounding of the proposal: the shift moves the new angle by about 2.4e-7
(log_p by beta deg 2.4e-7 < 1e-5 here).  SU(N) decides in FP32: its staple
arithmetic and its candidate U exp(iX) (about 1e-6 per entry) each move log_p
by up to about (beta/N) N^2 deg 1e-6, 1e-4 at beta 2.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5
MARGIN_U1 = 2e-5
MARGIN_SU = 2e-4


def _setup(umc, oracle, cc):
    _, _, pos = cc.colouring()
    cells = cc.table()
    rcells = pos[cells]
    inc = oracle.cell_incidence(cc.sites(), rcells)[1:]
    return pos, rcells, inc


def _cell_neighbours(cells, links):
    links = set(links)
    out = set()
    for c in cells:
        if links & set(c.tolist()):
            out.update(c.tolist())
    return out


def _su_field(ch, N):
    f = ch.get_field().reshape(-1, N, N, 2).astype(np.float64)
    return f[..., 0] + 1j * f[..., 1]


def _su_host(u):
    return np.stack([u.real, u.imag], axis=-1).astype(np.float32).reshape(len(u), -1)


@pytest.mark.parametrize("kind,L,beta,width,hits", [("2d", 8, 2.0, 0.5, 2), ("4d", 4, 1.1, 0.7, 1),
                                                     ("4d", 3, 0.9, 0.7, 3), ("2d", 5, 3.0, 1.0, 1)])
def test_u1_per_sweep(umc, oracle, kind, L, beta, width, hits):
    cc = umc.square_plaquettes(L) if kind == "2d" else umc.hypercubic_plaquettes(L)
    n = cc.sites()
    pos, rcells, inc = _setup(umc, oracle, cc)
    ch = umc.Chain(umc.MODEL_U1, cells=cc, coupling=beta, proposal=umc.PROPOSAL_U1SHIFT, width=width,
                   hits=hits, seed=3)
    th = np.random.default_rng(L).uniform(-np.pi, np.pi, n).astype(np.float32)
    ch.set_field(th)
    cells_site = cc.table()
    mism = 0
    for sweep in range(3):
        state = ch.get_field().astype(np.float64)
        cm = np.empty(n)
        cm[pos] = state
        t_o, obs_o, margin = oracle.u1_metropolis(rcells, inc, beta, 1.0, width, hits, 3, sweep, 1, cm)
        rec = ch.metropolis(1.0, 1)
        got = ch.get_field().astype(np.float64)
        d = np.abs(np.angle(np.exp(1j * (got - t_o[pos]))))
        bad = np.nonzero(d > TOL)[0]
        near = np.nonzero(np.abs(margin[pos]) < MARGIN_U1)[0]
        assert set(bad.tolist()) <= _cell_neighbours(cells_site, near) | set(near.tolist()), (bad, d[bad])
        mism += len(bad)
        P_true = oracle.u1_mean_plaquette(cells_site, got)
        assert abs(rec[0, 1] - P_true) < 1e-6
        assert abs(rec[0, 0] - beta * len(cells_site) * (1 - P_true)) < 1e-4 * max(1.0, abs(rec[0, 0]))
        if kind == "2d":
            assert abs(rec[0, 2] - oracle.u1_topological_charge(cells_site, got)) < 1e-4
    assert mism <= max(2, n // 50)


@pytest.mark.parametrize("N,L,hits", [(3, 2, 2), (2, 4, 1), (3, 3, 1), (3, 3, 10), (2, 2, 10)])
def test_su_per_sweep(umc, oracle, N, L, hits):
    """hits = 10 is the SU(3) configuration's multi-hit count: ten proposals
    per link in a row, each from its own keyed stream."""
    cc = umc.hypercubic_plaquettes(L)
    n = cc.sites()
    pos, rcells, inc = _setup(umc, oracle, cc)
    beta, width = 2.0, 0.3
    ch = umc.Chain(umc.MODEL_SU, cells=cc, components=N, coupling=beta, proposal=umc.PROPOSAL_SUSHIFT,
                   width=width, hits=hits, seed=11)
    ch.randomize(5)
    cells_site = cc.table()
    mism = 0
    for sweep in range(2):
        u = _su_field(ch, N)
        cm = np.empty_like(u)
        cm[pos] = u
        u_o, obs_o, margin = oracle.su_metropolis(N, rcells, inc, beta, 1.0, width, hits, 11, sweep, 1, cm)
        rec = ch.metropolis(1.0, 1)
        got = _su_field(ch, N)
        d = np.abs(got - u_o[pos]).reshape(n, -1).max(axis=1)
        bad = np.nonzero(d > TOL)[0]
        near = np.nonzero(np.abs(margin[pos]) < MARGIN_SU)[0]
        assert set(bad.tolist()) <= _cell_neighbours(cells_site, near) | set(near.tolist()), (bad, d[bad])
        mism += len(bad)
        P_true = oracle.su_mean_plaquette(N, cells_site, got)
        assert abs(rec[0, 1] - P_true) < 2e-6
        for k in range(0, n, max(1, n // 16)):
            assert oracle.su_unitarity_error(N, got[k]) < 2e-6
    assert mism <= max(2, n // 50)


def test_su3_haar_start(umc):
    cc = umc.hypercubic_plaquettes(8)
    ch = umc.Chain(umc.MODEL_SU, cells=cc, components=3, coupling=5.7, proposal=umc.PROPOSAL_SUSHIFT, width=0.2,
                   hits=1, seed=1)
    ch.randomize(123)
    u = _su_field(ch, 3)
    assert np.abs(np.einsum("nji,njk->nik", u.conj(), u) - np.eye(3)).max() < 2e-6
    assert np.abs(np.linalg.det(u) - 1).max() < 2e-6
    tr = np.trace(u, axis1=1, axis2=2)
    # Haar moments: E Tr U = 0, E |Tr U|^2 = 1
    assert abs(tr.mean()) < 0.03
    assert abs((np.abs(tr) ** 2).mean() - 1.0) < 0.05
    ch.randomize(123)
    np.testing.assert_array_equal(_su_field(ch, 3), u)


def test_gauge_limits(umc):
    # test/u1_check.cpp:78-95 and test/su_check.cpp:102-135, beta placed once
    cc = umc.hypercubic_plaquettes(4)
    ch = umc.Chain(umc.MODEL_U1, cells=cc, coupling=0.0, proposal=umc.PROPOSAL_U1SHIFT, width=0.7, seed=10)
    rec = ch.metropolis(1.0, 300)
    assert abs(rec[100:, 1].mean()) < 0.05
    ch = umc.Chain(umc.MODEL_U1, cells=cc, coupling=10.0, proposal=umc.PROPOSAL_U1SHIFT, width=0.7, seed=20)
    rec = ch.metropolis(1.0, 300)
    assert rec[100:, 1].mean() > 0.9
    ch = umc.Chain(umc.MODEL_SU, cells=cc, components=2, coupling=10.0, proposal=umc.PROPOSAL_SUSHIFT,
                   width=0.3, seed=50)
    rec = ch.metropolis(1.0, 300)
    assert rec[100:, 1].mean() > 0.9
    # hot and cold starts agree (SU(2), beta = 2, L = 4)
    hot = umc.Chain(umc.MODEL_SU, cells=cc, components=2, coupling=2.0, proposal=umc.PROPOSAL_SUSHIFT, width=0.3, seed=30)
    hot.randomize(9)
    cold = umc.Chain(umc.MODEL_SU, cells=cc, components=2, coupling=2.0, proposal=umc.PROPOSAL_SUSHIFT, width=0.3, seed=40)
    a = hot.metropolis(1.0, 600)[200:, 1].mean()
    b = cold.metropolis(1.0, 600)[200:, 1].mean()
    assert abs(a - b) < 0.03


def test_su3_long_chain_stays_unitary(umc):
    cc = umc.hypercubic_plaquettes(6)
    ch = umc.Chain(umc.MODEL_SU, cells=cc, components=3, coupling=5.7, proposal=umc.PROPOSAL_SUSHIFT, width=0.2,
                   hits=10, seed=7)
    ch.randomize(1)
    rec = ch.metropolis(1.0, 50)
    u = _su_field(ch, 3)
    assert np.abs(np.einsum("nji,njk->nik", u.conj(), u) - np.eye(3)).max() < 5e-6
    assert np.isfinite(rec).all()
    assert rec[-1, 1] > rec[0, 1]  # ordering from the hot start at beta 5.7
    assert rec[:, 7].sum() > 0
