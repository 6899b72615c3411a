"""Streaming Gamma-method sums on the host: chunking does not matter and the
result equals the full-series Gamma-method (restated from critmc's
stats/autocorr.py:381, pinned in test_oracle_stats)."""

from __future__ import annotations

import numpy as np
import pytest
from exact_helpers import ar1, gamma_error

from critmc_b200.streaming import HostStreamStats


@pytest.mark.parametrize("phi,n", [(0.0, 3000), (0.6, 20000), (0.9, 50000)])
def test_streaming_equals_full_series(phi, n):
    x = ar1(7, phi, n) * 3.0 + 100.0
    rng = np.random.default_rng(1)
    cuts = np.sort(rng.integers(0, n, 25))
    hs = HostStreamStats(max_lag=256)
    for part in np.split(x, cuts):
        hs.update(part)
    res = hs.result()
    mean, err, tau = gamma_error(x)
    assert res["n"] == n and not res["truncated"]
    assert res["mean"] == pytest.approx(mean, rel=1e-12, abs=1e-12)
    assert res["error"] == pytest.approx(err, rel=1e-8)
    assert res["tau_int"] == pytest.approx(tau, rel=1e-8)


def test_chunking_does_not_matter_and_integers_work():
    x = np.cumsum(np.random.default_rng(3).integers(-5, 6, 4000)).astype(np.int64) - 12345678
    a, b = HostStreamStats(64), HostStreamStats(64)
    a.update(x)
    for i in range(0, x.size, 333):
        b.update(x[i:i + 333])
    np.testing.assert_allclose(a.state, b.state, rtol=1e-12, atol=1e-6)
    assert a.result()["truncated"]  # a random walk needs a longer window than 64


def test_short_and_constant_series():
    hs = HostStreamStats(16)
    hs.update([5.0])
    r = hs.result()
    assert r["n"] == 1 and r["mean"] == 5.0
    hs.update(np.full(100, 5.0))
    r = hs.result()
    assert r["error"] == 0.0 and r["mean"] == 5.0
