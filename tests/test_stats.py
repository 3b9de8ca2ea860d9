"""Force statistics (js/main.js:59-212) on the host: checked against the formulas
written out independently here, on synthetic force series (no GPU)."""
import math

import numpy as np
import pytest

from windtunnel_b200 import stats


def test_block_stats_short_series_is_plain_sem():
    x = np.array([1.0, 2.0, 4.0, 7.0, 11.0])
    b = stats.block_stats(x)
    assert not b.blocked
    assert b.mean == pytest.approx(x.mean())
    assert b.sem == pytest.approx(x.std(ddof=1) / math.sqrt(len(x)))


def test_block_stats_uses_16_blocks():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(16 * 37 + 5)
    b = stats.block_stats(x)
    assert b.blocked and b.used == 16 * 37
    bm = x[: 16 * 37].reshape(16, 37).mean(axis=1)
    assert b.mean == pytest.approx(bm.mean())
    assert b.sem == pytest.approx(bm.std(ddof=1) / 4.0)


def odd_even_series(n, mean=(3.0, 0.5, -0.2), amp=1.5, seed=1):
    """A force series with the lattice's odd/even oscillation plus noise."""
    rng = np.random.default_rng(seed)
    s = np.sign(np.cos(np.pi * np.arange(n)))[:, None]
    return np.array(mean)[None, :] + amp * s + 0.01 * rng.standard_normal((n, 3))


def test_pair_averaging_cancels_the_parity_oscillation():
    F = odd_even_series(1000)
    u0, area = 0.05, 144
    q = 0.5 * u0 * u0 * area
    st = stats.ForceStats(u0=u0, ref_area=area, settle=10)
    for f in F:
        st.accumulate(f)
    r = st.run_stats()
    # 10 settle steps, then the first sample only primes prevF
    assert r.n == 1000 - 10 - 1
    assert r.cd.mean == pytest.approx(3.0 / q, rel=1e-3)
    assert r.cl.mean == pytest.approx(0.5 / q, rel=1e-2)
    raw = F[11:, 0] / q
    assert r.cd.sem < 0.05 * raw.std()          # the oscillation is gone
    assert r.state in ("converged", "noisy")


def test_ring_keeps_the_last_hist_samples_in_order():
    n = stats.HIST + 250
    F = np.zeros((n + 2, 3))
    F[:, 0] = np.arange(n + 2, dtype=float)
    st = stats.ForceStats(u0=1.0, ref_area=2.0, settle=0)
    for f in F:
        st.accumulate(f)
    x = st.ordered(st.h_cd)
    assert len(x) == stats.HIST
    assert np.all(np.diff(x) > 0)
    # pair average of the last two forces over q = 0.5*1*1*2 = 1
    assert x[-1] == pytest.approx(0.5 * (F[-1, 0] + F[-2, 0]), rel=1e-6)
    # float32 ring, as the reference's Float32Array history
    assert st.h_cd.dtype == np.float32


def test_drift_is_flagged():
    n = 2000
    F = np.zeros((n, 3))
    F[:, 0] = 1.0 + np.linspace(0, 0.5, n)     # a slow trend
    r = stats.series_stats(F, u0=1.0, ref_area=2.0, settle=0)
    assert r.state == "drifting"
    assert r.drift > 2.5 * r.cd.sem


def test_too_short_run_has_no_stats():
    assert stats.series_stats(np.ones((50, 3)), 0.05, 10, settle=0) is None


def test_ema_matches_reference_update():
    st = stats.ForceStats(u0=1.0, ref_area=1.0, settle=0)
    ema = [0.0, 0.0, 0.0]
    rng = np.random.default_rng(3)
    for k in range(1, 700):
        f = rng.standard_normal(3)
        st.accumulate(f)
        a = 1 / min(k, 500)
        ema = [e + (fk - e) * a for e, fk in zip(ema, f)]
    assert np.allclose(st.force_ema, ema)


def test_window_coefficients_match_series_pipeline():
    F = odd_even_series(4000, seed=7)
    w = stats.window_coefficients(F, 0.06, 100, 2000)
    q = 0.5 * 0.06 ** 2 * 100
    pa = 0.5 * (F[1:] + F[:-1])[-2000:] / q
    assert w["cd"] == pytest.approx(pa[:, 0].mean())
    assert w["cd_sem"] > 0
