"""Device streaming Gamma-method sums: the same state as the host restatement,
slice after slice, for int64 and double series of many chains."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from exact_helpers import ar1, gamma_error

from critmc_b200.ensemble import IsingEnsemble
from critmc_b200.streaming import HostStreamStats, StreamStats

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [torch.float64, torch.int64])
@pytest.mark.parametrize("W", [8, 100, 256])
def test_device_state_equals_host(cuda, dtype, W):
    n_chains, n = 5, 5000
    if dtype == torch.float64:
        x = np.stack([ar1(c, 0.7, n) * 2.0 + c for c in range(n_chains)])
    else:
        x = np.stack([np.cumsum(np.random.default_rng(c).integers(-3, 4, n)) - 1000 * c for c in range(n_chains)])
    dev = StreamStats(n_chains, W, cuda)
    hosts = [HostStreamStats(W) for _ in range(n_chains)]
    for lo, hi in ((0, 1), (1, 7), (7, 2500), (2500, 2501), (2501, n)):
        dev.update(torch.from_numpy(np.ascontiguousarray(x[:, lo:hi])).to(cuda, dtype))
        for c in range(n_chains):
            hosts[c].update(x[c, lo:hi])
    st = dev.state.cpu().numpy().reshape(n_chains, -1)
    for c in range(n_chains):
        np.testing.assert_allclose(st[c], hosts[c].state, rtol=1e-11, atol=1e-6)
        r, h = dev.result()[c], hosts[c].result()
        assert r["window"] == h["window"]
        assert r["error"] == pytest.approx(h["error"], rel=1e-9)


def test_ensemble_series_error_bars_without_host_series(cuda):
    ens = IsingEnsemble(128, (0.40, 0.44), 4, seed=6, device=cuda)
    ens.run(200, host=False)
    stats = StreamStats(ens.n_chains, 256, cuda)
    kept = []
    for _ in range(5):
        out = ens.run(1000, host=False)
        stats.update(out.Eb)
        kept.append(out.Eb.cpu().numpy())
    series = np.concatenate(kept, axis=1)
    for c, r in enumerate(stats.result()):
        mean, err, tau = gamma_error(series[c].astype(np.float64))
        assert r["mean"] == pytest.approx(mean, rel=1e-12)
        if not r["truncated"]:
            assert r["error"] == pytest.approx(err, rel=1e-7)
            assert r["tau_int"] == pytest.approx(tau, rel=1e-7)
