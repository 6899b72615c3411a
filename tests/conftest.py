from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long statistical runs")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device; GPU tests fail (not skip) when it is missing."""
    import torch

    assert torch.cuda.is_available(), "the gpu tests need a CUDA device"
    return torch.device("cuda", 0)


def batch_mean_error(x: np.ndarray, n_batches: int = 64) -> tuple[float, float]:
    """Mean of the series, and its standard error from ``n_batches`` equal blocks
    after dropping the leading remainder (the statistic of critmc tests/conftest.py:6-11)."""
    series = np.asarray(x, dtype=np.float64)
    drop = series.size % n_batches
    block_means = series[drop:].reshape(n_batches, -1).mean(axis=1)
    return float(series.mean()), float(np.std(block_means, ddof=1) / np.sqrt(n_batches))


def assert_consistent(sample, exact: float, z_max: float = 4.5, n_batches: int = 64):
    """The sample mean lies within ``z_max`` batch-means errors of ``exact``
    (critmc tests/conftest.py:14-17 uses 4.5)."""
    mean, err = batch_mean_error(sample, n_batches)
    z = 0.0 if err <= 0 else (mean - exact) / err
    assert abs(z) < z_max, f"sample mean {mean:.6g} +- {err:.2g} is {z:+.2f} errors from {exact:.6g}"
