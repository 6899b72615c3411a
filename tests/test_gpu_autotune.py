"""Autotuner on the GPU: its choices are valid and change no result."""

from __future__ import annotations

import numpy as np
import pytest

from critmc_b200 import autotune
from critmc_b200.ensemble import IsingEnsemble

pytestmark = pytest.mark.gpu


@pytest.fixture
def tune_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("CRITMC_B200_TUNE_CACHE", str(tmp_path / "tune.json"))


def test_tuned_ensemble_gives_the_same_series(cuda, tune_cache):
    a = IsingEnsemble(256, (0.42, 0.45), 3, seed=4, device=cuda)
    b = IsingEnsemble(256, (0.42, 0.45), 3, seed=4, device=cuda, tune=True)
    assert b.tuning["run"] in autotune.MSC_RUNS and b.tuning["k_inline"] in (4, 8)
    ra, rb = a.run(20), b.run(20)
    np.testing.assert_array_equal(ra.Eb, rb.Eb)
    np.testing.assert_array_equal(ra.M, rb.M)
    np.testing.assert_array_equal(ra.aux, rb.aux)
    assert autotune.tune_msc((256, 256), 6, device=cuda) == b.tuning  # served from the cache


@pytest.mark.parametrize("run", autotune.MSC_RUNS)
def test_every_rows_per_thread_choice_gives_the_same_series(cuda, run):
    ref = IsingEnsemble(128, (0.44,), 2, seed=2, device=cuda)
    alt = IsingEnsemble(128, (0.44,), 2, seed=2, device=cuda, mode=autotune.msc_mode(run, 1), k_inline=4)
    for n in (3, 5):
        x, y = ref.run(n, "metropolis+heatbath"), alt.run(n, "metropolis+heatbath")
        np.testing.assert_array_equal(x.Eb, y.Eb)
        np.testing.assert_array_equal(x.M, y.M)


def test_on_grid_and_serving_calibration(cuda, tune_cache):
    best = autotune.tune_on_grid((64, 64), 2, n_meas=16, device=cuda)
    assert best["blocks_per_chain"] >= 1
    costs = autotune.calibrate_serving(cuda, n_meas=20)
    assert set(costs) == set(autotune._SERVE_PROBES)
    assert all(a > 0 and b >= 0 for a, b in costs.values())
