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
    """Mean and batch-means standard error (critmc tests/conftest.py:6-11)."""
    x = np.asarray(x, dtype=np.float64)
    size = len(x) // n_batches
    b = x[len(x) - size * n_batches:].reshape(n_batches, size).mean(axis=1)
    return float(x.mean()), float(b.std(ddof=1) / np.sqrt(n_batches))


def assert_consistent(sample, exact: float, z_max: float = 4.5, n_batches: int = 64):
    """|z| < z_max with batch-means errors (critmc tests/conftest.py:14-17)."""
    mean, err = batch_mean_error(sample, n_batches)
    z = (mean - exact) / err if err > 0 else 0.0
    assert abs(z) < z_max, f"mean {mean:.6f} +- {err:.2e} vs exact {exact:.6f} (z = {z:.2f})"
