"""Runner on the GPU (critmc runner.py:87-195): tasks run through Simulation,
results written to and reloaded from the cache, identical to a direct run."""

from __future__ import annotations

import numpy as np
import pytest

from critmc_b200.runner import Task, run_task, run_tasks
from critmc_b200.sim import TimeSeries

pytestmark = pytest.mark.gpu

TASKS = [
    Task({"model": "ising", "lattice": "square", "L": 16}, 0.44, "metropolis", 50, 200, 7, keys=("i", 0)),
    Task({"model": "potts", "lattice": "square", "L": 8, "q": 3}, 1.0, "heatbath+sw", 20, 100, 7, keys=("p",)),
    Task({"model": "on", "lattice": "square", "L": 8, "n": 2}, 1.1, "heatbath+2*overrelax+wolff", 20, 50, 7,
         name="xy8"),
]


def test_run_tasks_caches_and_reloads(cuda, tmp_path):
    first = run_tasks(TASKS, out_dir=tmp_path, progress=False)
    files = sorted(p.name for p in tmp_path.iterdir())
    assert files == sorted(t.filename for t in TASKS)
    again = run_tasks(TASKS, out_dir=tmp_path, progress=False)
    for a, b, t in zip(first, again, TASKS):
        assert set(a.raw) == set(b.raw)
        for k in a.raw:
            np.testing.assert_array_equal(a.raw[k], b.raw[k])
        assert b.meta["task"]["seed"] == t.seed
    # the files are critmc's format: TimeSeries.load reads them back
    ts = TimeSeries.load(tmp_path / TASKS[0].filename)
    assert ts.raw["E"].shape == (200,)


def test_run_task_is_reproducible(cuda):
    a = run_task(TASKS[0])
    b = run_tasks([TASKS[0]], progress=False)[0]
    np.testing.assert_array_equal(a.raw["E"], b.raw["E"])
    np.testing.assert_array_equal(a.raw["M"], b.raw["M"])
    assert a.meta["task"]["keys"] == ("i", 0)
