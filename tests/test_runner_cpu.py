"""Task cache of the runner on the CPU (critmc runner.py:33-109, 154-195):
file names, reuse of a result written by the same task, StaleCacheError for
a file from another task, and the order-preserving host map."""

from __future__ import annotations

import math
from dataclasses import asdict

import numpy as np
import pytest

from critmc_b200.runner import StaleCacheError, Task, parallel_map, run_tasks
from critmc_b200.sim import TimeSeries

SPEC = {"model": "ising", "lattice": "square", "L": 8}


def _task(**kw) -> Task:
    base = dict(model=SPEC, beta=0.44, updates="metropolis", n_therm=10, n_meas=20, seed=3, keys=("a", 1))
    base.update(kw)
    return Task(**base)


def _cached(task: Task, d, meta_task=True) -> TimeSeries:
    meta = {"model": "ising", "N": 64, "beta": task.beta}
    if meta_task:
        meta["task"] = asdict(task)
    ts = TimeSeries({"E": np.arange(task.n_meas, dtype=np.float64), "Eb": np.arange(task.n_meas)}, meta)
    ts.save(d / task.filename)
    return ts


def test_task_filenames():
    assert _task().filename == "ising_L8_b0.44000000_a_1.npz"
    assert _task(keys=()).filename == "ising_L8_b0.44000000_run.npz"
    assert _task(name="x").filename == "x.npz"


def test_cached_result_is_reused_without_running(tmp_path):
    t = _task()
    ref = _cached(t, tmp_path)
    (tmp_path / "left.part.npz").write_bytes(b"partial")
    out = run_tasks([t], out_dir=tmp_path, progress=False)
    np.testing.assert_array_equal(out[0].raw["E"], ref.raw["E"])
    assert out[0].meta["task"]["keys"] == ["a", 1]
    assert not (tmp_path / "left.part.npz").exists()


def test_file_from_another_task_is_stale(tmp_path):
    _cached(_task(seed=4), tmp_path)
    with pytest.raises(StaleCacheError, match="seed"):
        run_tasks([_task()], out_dir=tmp_path, progress=False)


def test_file_without_a_task_record_is_stale(tmp_path):
    _cached(_task(), tmp_path, meta_task=False)
    with pytest.raises(StaleCacheError, match="does not record"):
        run_tasks([_task()], out_dir=tmp_path, progress=False)


def test_parallel_map_keeps_order():
    items = list(range(1, 40))
    assert parallel_map(math.sqrt, items, workers=3, progress=False) == [math.sqrt(i) for i in items]
    assert parallel_map(abs, [-2, 1], workers=1, progress=False) == [2, 1]
