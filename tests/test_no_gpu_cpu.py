"""Without a GPU the product fails loudly: no CPU fallback on any public entry point
(the CPU oracle is test infrastructure only)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from critmc_b200 import ON, Ising, Potts, Simulation, square

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error")


@pytest.mark.parametrize("make", [lambda: Simulation(Ising(square(64)), 0.44, seed=1),
                                  lambda: Simulation(Ising(square(6)), 0.44, seed=1),
                                  lambda: Simulation(Potts(square(4), 3), 1.0, seed=1),
                                  lambda: Simulation(ON(square(8), 2), 1.0, "heatbath", seed=1)],
                         ids=["ising-msc", "ising-byte", "potts", "xy"])
def test_simulation_needs_a_gpu(make):
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        make()


def test_batched_and_flat_histogram_drivers_need_a_gpu():
    from critmc_b200.ensemble import IsingEnsemble
    from critmc_b200.flathist import Multicanonical, WangLandau

    with pytest.raises(RuntimeError, match="no CPU fallback"):
        IsingEnsemble(64, [0.44], 2, seed=1)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        WangLandau(Ising(square(4)), seed=1)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        Multicanonical(Ising(square(4)), np.zeros(17), seed=1)


def test_runner_needs_a_gpu_for_pending_tasks(tmp_path):
    from critmc_b200.runner import Task, run_tasks

    task = Task({"model": "ising", "lattice": "square", "L": 8}, 0.44, "metropolis", 1, 1, 1)
    with pytest.raises((RuntimeError, AssertionError)):
        run_tasks([task], out_dir=tmp_path, progress=False)
