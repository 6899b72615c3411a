"""Resumable execution of simulation batches on the GPU (critmc ``runner``).

A :class:`Task` names one chain: model spec, beta, update string, run lengths,
and a random stream derived from ``(seed, *keys)``, so each task gives the
same result whatever runs it and in which order.  With ``out_dir``, every
result goes to ``<out_dir>/<task.filename>`` as soon as it is done, in the
series format of :mod:`critmc_b200.io`, which is critmc's: those files load with
critmc's ``TimeSeries.load``, and critmc's own caches load here.  A later call
with the same ``out_dir`` reuses the files of tasks that are done; a file that
records a different task raises :class:`StaleCacheError` before anything runs.

critmc spreads pending tasks over a process pool, one chain per core
(``runner.py:154-195``).  Here the sweeps run on the GPU, so the workers are
the visible GPUs: one host thread per device takes the next pending task (the
library calls release the GIL).  :func:`parallel_map` stays a process pool for
host functions.
"""

from __future__ import annotations

import multiprocessing as mp
import os
import queue
import sys
import threading
import time
from collections.abc import Callable, Iterable, Sequence
from concurrent.futures import ProcessPoolExecutor
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Any

from .io import to_jsonable
from .models import build_model
from .rng import make_rng
from .sim import Simulation, TimeSeries

__all__ = ["Task", "StaleCacheError", "run_task", "run_tasks", "parallel_map", "default_workers"]

WORKER_BYTES = 1 << 30  # host memory one parallel_map worker may need


@dataclass(frozen=True)
class Task:
    """One chain to run (critmc runner.py:33-56); ``model`` is a spec for ``build_model``."""

    model: dict[str, Any]
    beta: float
    updates: str
    n_therm: int
    n_meas: int
    seed: int
    keys: tuple = ()
    start: str = "random"
    name: str = ""
    extra: dict[str, Any] = field(default_factory=dict)

    @property
    def filename(self) -> str:
        """``<name>.npz``, else ``<model>_L<L>_b<beta, 8 decimals>_<keys joined by _ or 'run'>.npz``."""
        if self.name:
            return self.name + ".npz"
        keys = "_".join(map(str, self.keys)) if self.keys else "run"
        return "{}_L{}_b{:.8f}_{}.npz".format(self.model["model"], self.model["L"], self.beta, keys)


class StaleCacheError(ValueError):
    """A cached result file was produced by a different task than the one requested."""


def _record(task: Task) -> dict[str, Any]:
    """The task as its result file stores it (JSON conventions of the series format)."""
    return to_jsonable(asdict(task))


def _reuse(task: Task, path: Path) -> TimeSeries:
    """The cached result of ``task`` at ``path``, after checking the file is really its."""
    ts = TimeSeries.load(path)
    stored = ts.meta.get("task")
    wanted = _record(task)
    if stored == wanted:
        return ts
    if isinstance(stored, dict):
        why = "; ".join(f"{key}: file has {stored.get(key)!r}, requested {value!r}"
                        for key, value in wanted.items() if stored.get(key) != value)
    else:
        why = "it does not record the task that produced it"
    raise StaleCacheError(f"{path} was not produced by the requested task ({why}); "
                          "pick another out_dir or remove the file")


def run_task(task: Task, device=None) -> TimeSeries:
    """Thermalise and run one task on ``device`` (critmc runner.py:87-95)."""
    sim = Simulation(build_model(task.model), task.beta, task.updates, seed=make_rng(task.seed, *task.keys),
                     start=task.start, device=device)
    sim.thermalize(task.n_therm)
    ts = sim.run(task.n_meas)
    ts.meta["task"] = asdict(task)
    ts.meta["tuning"] = sim.tuning()
    return ts


def _run_and_store(task: Task, out: Path | None, device=None) -> TimeSeries:
    ts = run_task(task, device)
    if out is None:
        return ts
    final = out / task.filename
    partial = final.with_suffix(".part.npz")  # renamed into place only once complete
    ts.save(partial)
    os.replace(partial, final)
    return TimeSeries.load(final)


def default_workers() -> int:
    """Host processes for :func:`parallel_map`: the cores but one, and no more than the
    free memory holds at ``WORKER_BYTES`` each (at least one)."""
    n = (os.cpu_count() or 2) - 1
    try:
        import psutil

        n = min(n, int(psutil.virtual_memory().available // WORKER_BYTES) - 1)
    except (ImportError, OSError):
        pass
    return max(1, n)


class _Progress:
    def __init__(self, total: int, enabled: bool):
        self.total, self.enabled, self.done, self.t0 = total, enabled, 0, time.perf_counter()
        self.lock = threading.Lock()

    def step(self) -> None:
        with self.lock:
            self.done += 1
            if not self.enabled:
                return
            spent = time.perf_counter() - self.t0
            left = spent / self.done * (self.total - self.done)
            end = "\n" if self.done == self.total else ""
            sys.stderr.write(f"\r  {self.done}/{self.total} done, {spent:.1f} s, about {left:.1f} s to go{end}")
            sys.stderr.flush()


def _visible_gpus() -> list[int]:
    import torch

    return list(range(torch.cuda.device_count())) if torch.cuda.is_available() else [0]


def run_tasks(tasks: Sequence[Task], *, workers: int | None = None, out_dir: str | Path | None = None,
              progress: bool = True, devices: Sequence[int] | None = None) -> list[TimeSeries]:
    """Results of ``tasks`` in task order (critmc runner.py:154-195).

    With ``out_dir``, finished tasks are read from their files (a file of another
    task raises :class:`StaleCacheError` first) and the others are written there.
    The pending tasks go to one thread per device of ``devices`` (default: the
    visible GPUs, at most ``workers`` of them).
    """
    out = Path(out_dir) if out_dir is not None else None
    if out is not None:
        out.mkdir(parents=True, exist_ok=True)
        for leftover in out.glob("*.part.npz"):  # from a run that was interrupted
            leftover.unlink()
    results: list[TimeSeries | None] = [None] * len(tasks)
    todo: queue.Queue[int] = queue.Queue()
    for i, task in enumerate(tasks):
        cached = out / task.filename if out is not None else None
        if cached is not None and cached.exists():
            results[i] = _reuse(task, cached)
        else:
            todo.put(i)
    n_todo = todo.qsize()
    if n_todo:
        gpus = list(devices) if devices is not None else _visible_gpus()
        if workers is not None:
            gpus = gpus[: max(1, int(workers))]
        meter = _Progress(n_todo, progress)
        failures: list[BaseException] = []

        def serve(dev: int) -> None:
            import torch

            torch.cuda.set_device(dev)
            while not failures:
                try:
                    i = todo.get_nowait()
                except queue.Empty:
                    return
                try:
                    results[i] = _run_and_store(tasks[i], out, device=f"cuda:{dev}")
                except BaseException as err:  # noqa: BLE001 - raised again by the caller
                    failures.append(err)
                    return
                meter.step()

        threads = [threading.Thread(target=serve, args=(d,), daemon=True) for d in gpus[1:]]
        for th in threads:
            th.start()
        serve(gpus[0])  # the calling thread serves the first device
        for th in threads:
            th.join()
        if failures:
            raise failures[0]
    return results  # type: ignore[return-value]


def parallel_map(fn: Callable, items: Iterable, *, workers: int | None = None, progress: bool = True) -> list:
    """``[fn(x) for x in items]`` over a process pool (critmc runner.py:198-220).

    ``fn`` must be a picklable top-level function.  The pool starts its
    processes with ``spawn``: a process forked from one that has used CUDA
    cannot use it.
    """
    work = list(items)
    n = default_workers() if workers is None else max(1, int(workers))
    meter = _Progress(len(work), progress)
    if n == 1 or len(work) <= 1:
        out = []
        for x in work:
            out.append(fn(x))
            meter.step()
        return out
    out = []
    with ProcessPoolExecutor(max_workers=min(n, len(work)), mp_context=mp.get_context("spawn")) as pool:
        for value in pool.map(fn, work):
            out.append(value)
            meter.step()
    return out
