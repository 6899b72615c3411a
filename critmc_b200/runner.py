"""Resumable execution of simulation batches on the GPU (critmc ``runner``).

API of critmc ``src/critmc/runner.py``: a :class:`Task` describes one chain,
its random stream comes from ``(seed, *keys)``, and with an output directory
each result is written to ``<dir>/<name>.npz`` as soon as it is done (in
critmc's ``.npz`` + JSON format, so critmc's own ``TimeSeries.load`` and the
pipelines behind it read it).  Tasks whose file exists are loaded instead of
run.  A file left by a different task raises :class:`StaleCacheError`.

critmc runs pending tasks in a process pool, one chain per core.  Here a
chain's sweeps run on the GPU, so the workers of :func:`run_tasks` are GPUs:
one host thread per device, each running its share of the tasks through the
GPU :class:`~critmc_b200.sim.Simulation` (the library calls release the GIL).
A task's result does not depend on which device or thread ran it.
:func:`parallel_map` stays a process pool for arbitrary host functions.
"""

from __future__ import annotations

import multiprocessing as mp
import os
import sys
import threading
import time
from collections.abc import Callable, Iterable, Sequence
from concurrent.futures import ProcessPoolExecutor, as_completed
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Any

from .io import to_jsonable
from .models import build_model
from .rng import make_rng
from .sim import Simulation, TimeSeries

__all__ = ["Task", "StaleCacheError", "run_task", "run_tasks", "parallel_map", "default_workers"]


@dataclass(frozen=True)
class Task:
    """One canonical Markov chain (critmc runner.py:33-56).

    ``model`` is a model spec such as ``{"model": "ising", "lattice": "square", "L": 32}``.
    """

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
        if self.name:
            return f"{self.name}.npz"
        tag = "_".join(str(k) for k in self.keys) or "run"
        return f"{self.model['model']}_L{self.model['L']}_b{self.beta:.8f}_{tag}.npz"


class StaleCacheError(ValueError):
    """A cached result file was produced by a different task than the one requested."""


def _task_record(task: Task) -> dict[str, Any]:
    return to_jsonable(asdict(task))


def _load_cached(task: Task, path: Path) -> TimeSeries:
    """Load a cached result after checking that ``task`` produced it (critmc runner.py:63-84)."""
    ts = TimeSeries.load(path)
    wanted = _task_record(task)
    found = ts.meta.get("task")
    if found == wanted:
        return ts
    if not isinstance(found, dict):
        detail = "it does not record the task that produced it"
    else:
        detail = "; ".join(f"{k}: file has {found.get(k)!r}, requested {wanted[k]!r}"
                           for k in wanted if found.get(k) != wanted[k])
    raise StaleCacheError(f"{path} was not produced by the requested task ({detail}). "
                          "Use a different out_dir or delete the file.")


def run_task(task: Task, device=None) -> TimeSeries:
    """Execute a task on ``device`` (critmc runner.py:87-95)."""
    model = build_model(task.model)
    rng = make_rng(task.seed, *task.keys)
    sim = Simulation(model, task.beta, task.updates, seed=rng, start=task.start, device=device)
    sim.thermalize(task.n_therm)
    ts = sim.run(task.n_meas)
    ts.meta.update({"task": asdict(task), "tuning": sim.tuning()})
    return ts


def _run_and_save(task: Task, out_dir: str | None, device=None) -> TimeSeries | str:
    ts = run_task(task, device)
    if out_dir is None:
        return ts
    path = Path(out_dir) / task.filename
    tmp = path.with_suffix(".part.npz")
    ts.save(tmp)
    os.replace(tmp, path)
    return str(path)


def _gpu_count() -> int:
    import torch

    return torch.cuda.device_count() if torch.cuda.is_available() else 0


_BYTES_PER_WORKER = 1 << 30


def _available_memory() -> int | None:
    try:
        return int(os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE"))
    except (AttributeError, OSError, ValueError):
        return None


def default_workers() -> int:
    """Host processes for :func:`parallel_map`: one per core minus one, capped by free memory."""
    workers = max(1, (os.cpu_count() or 2) - 1)
    avail = _available_memory()
    if avail is not None:
        workers = min(workers, max(1, avail // _BYTES_PER_WORKER - 1))
    return int(workers)


def run_tasks(tasks: Sequence[Task], *, workers: int | None = None, out_dir: str | Path | None = None,
              progress: bool = True, devices: Sequence[int] | None = None) -> list[TimeSeries]:
    """Run tasks and return their time series in task order (critmc runner.py:154-195).

    With ``out_dir`` results are cached on disk and existing files are reused; a
    file from a different task raises :class:`StaleCacheError` before anything
    runs.  ``devices`` (default: all visible GPUs, at most ``workers`` of them)
    are served by one thread each, taking the next pending task in order.
    """
    out = str(out_dir) if out_dir is not None else None
    if out is not None:
        Path(out).mkdir(parents=True, exist_ok=True)
        for stale in Path(out).glob("*.part.npz"):  # left behind by an interrupted run
            stale.unlink()
    results: dict[int, TimeSeries] = {}
    pending = []
    for i, t in enumerate(tasks):
        path = Path(out) / t.filename if out is not None else None
        if path is not None and path.exists():
            results[i] = _load_cached(t, path)
        else:
            pending.append(i)
    if not pending:
        return [results[i] for i in range(len(tasks))]
    if devices is None:
        devices = list(range(max(1, _gpu_count())))
    devices = list(devices)[: max(1, int(workers))] if workers is not None else list(devices)
    t0 = time.perf_counter()
    lock = threading.Lock()
    queue = list(pending)
    errors: list[BaseException] = []
    done = [0]

    def worker(dev: int) -> None:
        import torch

        torch.cuda.set_device(dev)
        while True:
            with lock:
                if not queue or errors:
                    return
                i = queue.pop(0)
            try:
                res = _run_and_save(tasks[i], out, device=f"cuda:{dev}")
                ts = TimeSeries.load(res) if isinstance(res, str) else res
            except BaseException as e:  # noqa: BLE001 - re-raised in the caller
                with lock:
                    errors.append(e)
                return
            with lock:
                results[i] = ts
                done[0] += 1
                if progress:
                    _report(done[0], len(pending), t0)

    if len(devices) == 1:
        worker(devices[0])
    else:
        threads = [threading.Thread(target=worker, args=(d,), daemon=True) for d in devices]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
    if errors:
        raise errors[0]
    return [results[i] for i in range(len(tasks))]


def parallel_map(fn: Callable, items: Iterable, *, workers: int | None = None, progress: bool = True) -> list:
    """Order-preserving parallel map of a picklable top-level host function (critmc runner.py:198-220).

    The pool starts its processes with ``spawn``: a process forked from one
    that has used CUDA cannot use it.
    """
    items = list(items)
    workers = default_workers() if workers is None else max(1, int(workers))
    t0 = time.perf_counter()
    if workers == 1 or len(items) <= 1:
        out = []
        for k, it in enumerate(items, 1):
            out.append(fn(it))
            if progress:
                _report(k, len(items), t0)
        return out
    results: dict[int, Any] = {}
    with ProcessPoolExecutor(max_workers=min(workers, len(items)), mp_context=mp.get_context("spawn")) as pool:
        futures = {pool.submit(fn, it): i for i, it in enumerate(items)}
        for k, fut in enumerate(as_completed(futures), 1):
            results[futures[fut]] = fut.result()
            if progress:
                _report(k, len(items), t0)
    return [results[i] for i in range(len(items))]


def _report(done: int, total: int, t0: float) -> None:
    elapsed = time.perf_counter() - t0
    eta = elapsed / done * (total - done)
    sys.stderr.write(f"\r  {done}/{total} done, {elapsed:7.1f}s elapsed, ~{eta:7.1f}s left")
    if done == total:
        sys.stderr.write("\n")
    sys.stderr.flush()
