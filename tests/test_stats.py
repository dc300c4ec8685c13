"""Host-side series statistics (umc_tau_int, umc_binning_error): exact agreement
with a numpy restatement, and the known integrated autocorrelation time of
AR(1) series, tau = (1 + rho) / (2 (1 - rho))."""
import numpy as np
import pytest


def _ar1(rho, n, seed):
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(n)
    x = np.empty(n)
    x[0] = e[0] / np.sqrt(1 - rho * rho)
    for i in range(1, n):
        x[i] = rho * x[i - 1] + e[i]
    return x


def _tau_numpy(x, c=6.0):
    d = x - x.mean()
    n = d.size
    c0 = d @ d / n
    t, w = 0.5, 0
    for w in range(1, n // 2 + 1):
        t += (d[:-w] @ d[w:]) / (n - w) / c0
        if w >= c * t:
            break
    return t, t * np.sqrt(2 * (2 * w + 1) / n), w


def test_tau_matches_numpy_restatement(umc):
    x = _ar1(0.7, 5000, 1)
    t, e, w = umc.tau_int(x)
    t2, e2, w2 = _tau_numpy(x)
    assert w == w2
    assert t == pytest.approx(t2, rel=1e-10)
    assert e == pytest.approx(e2, rel=1e-10)


@pytest.mark.parametrize("rho", [0.0, 0.5, 0.9, 0.95])
def test_tau_of_ar1(umc, rho):
    x = _ar1(rho, 200_000, 7)
    t, e, w = umc.tau_int(x)
    exact = (1 + rho) / (2 * (1 - rho))
    assert abs(t - exact) < 4 * e + 0.02 * exact, (t, e, exact)
    assert w >= 6 * t - 1


def test_binning_error_plateau_matches_tau(umc):
    rho = 0.8
    x = _ar1(rho, 400_000, 3)
    tau = (1 + rho) / (2 * (1 - rho))
    var = 1 / (1 - rho * rho)
    m, err = umc.binning_error(x, 2000)
    expect = np.sqrt(2 * tau * var / x.size)
    assert abs(m) < 5 * expect
    assert err == pytest.approx(expect, rel=0.15)
    m1, err1 = umc.binning_error(x, 1)
    assert m1 == pytest.approx(x[: x.size].mean(), rel=1e-12)
    assert err1 == pytest.approx(x.std(ddof=1) / np.sqrt(x.size), rel=1e-9)


def test_constant_series_and_errors(umc):
    t, e, w = umc.tau_int(np.ones(10))
    assert t == 0.5 and w == 0
    with pytest.raises(ValueError):
        umc.tau_int(np.ones(3))
    with pytest.raises(ValueError):
        umc.binning_error(np.ones(10), 6)
    with pytest.raises(ValueError):
        umc.binning_error(np.ones(10), 0)


def test_tau_multi_pools_chains(umc):
    rho = 0.8
    x = np.stack([_ar1(rho, 20_000, 100 + s) + s for s in range(16)])  # different means per chain
    t, e, w = umc.tau_int_multi(x)
    exact = (1 + rho) / (2 * (1 - rho))
    assert abs(t - exact) < 4 * e + 0.02 * exact, (t, e)
    t1, _, _ = umc.tau_int(x[3])
    assert abs(t1 - exact) < 0.2 * exact
    # frozen chains contribute nothing
    xf = np.concatenate([x, np.full((16, 20_000), 3.0)])
    tf, _, _ = umc.tau_int_multi(xf)
    assert tf == pytest.approx(t, rel=1e-9)
    assert umc.tau_int_multi(np.ones((3, 10)))[0] == 0.5


def test_observable_stream_round_trip_and_offline_tau(umc, tmp_path):
    """umc_obs_stream_*: records appended in chunks read back exactly, with
    the header's names, seed, first counter, model and beta; tau_int of the
    stored series equals tau_int of the series in memory; a partial read and
    reads beyond the stream behave."""
    rng = np.random.default_rng(4)
    phi, n = 0.8, 6000
    x = np.zeros(n)
    for t in range(1, n):
        x[t] = phi * x[t - 1] + rng.normal()
    rec = np.stack([x, x**2, np.arange(n, dtype=np.float64)], axis=1)
    path = tmp_path / "obs.umc"
    with umc.ObsStream(path, ["E", "E2", "sweep"], seed=17, first=1000, model=umc.MODEL_VECTOR, beta=0.693) as s:
        for k in range(0, n, 1024):
            s.append(rec[k:k + 1024])
        meta, mid = umc.read_obs_stream(path)  # readable while still open
        assert meta["records"] == n
    meta, got = umc.read_obs_stream(path)
    np.testing.assert_array_equal(got, rec)
    assert meta == {"names": ["E", "E2", "sweep"], "records": n, "seed": 17, "first": 1000,
                    "model": umc.MODEL_VECTOR, "beta": 0.693}
    assert umc.tau_int(got[:, 0]) == umc.tau_int(x)
    _, part = umc.read_obs_stream(path, first=10, n=5)
    np.testing.assert_array_equal(part, rec[10:15])
    with pytest.raises(IndexError):
        umc.read_obs_stream(path, first=n - 2, n=5)
    bad = tmp_path / "bad.umc"
    bad.write_bytes(b"not a stream at all, definitely not" * 3)
    with pytest.raises(ValueError):
        umc.read_obs_stream(bad)
