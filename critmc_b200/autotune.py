"""Autotuner for the launch shapes of the batched paths.

Every knob tuned here changes only how the work is laid out on the GPU, never
which random numbers a site sees, so any choice gives bit-identical results;
the tuner times the candidates on scratch copies of the workload's shape and
keeps the fastest.  Choices are cached in a JSON file keyed by (GPU name,
path, lattice shape, batch size, schedule, dtype): ``CRITMC_B200_TUNE_CACHE``
or ``~/.cache/critmc_b200/autotune.json``.

Tuned knobs:

* multi-spin-coded Ising (``critmc_ising_msc_run``): rows walked per thread
  (the column-walk tile height, 1..32) x acceptance planes resolved inline
  (``k_inline`` 4 or 8) x launch mode (one launch per half-sweep, or CUDA
  graphs replayed with a device cursor);
* O(n) multi-block lane (``critmc_on_run_grid``): thread blocks per chain;
* serving: the per-lane cost model (seconds per sweep = a + b * sites) of
  ``critmc_b200.serve.Server``, measured on one chain alone per lane.

critmc has no counterpart (its numba kernels have no launch shape).
"""

from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .device import empty_bytes, ptr, require_cuda, stream_handle, to_dev

MSC_RUNS = (1, 2, 4, 8, 16, 32)
MSC_K_INLINE = (4, 8)
MSC_MODES = (1, 3)


def cache_path() -> Path:
    p = os.environ.get("CRITMC_B200_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "critmc_b200" / "autotune.json"


def _load() -> dict:
    try:
        return json.loads(cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    data = _load()
    data[key] = value
    path = cache_path()
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(path)
    except OSError:
        pass  # a read-only home only loses the cache


def gpu_name(device) -> str:
    return torch.cuda.get_device_name(require_cuda(device))


def cache_key(device, path: str, shape, batch: int, schedule: str, dtype: str) -> str:
    return "|".join([gpu_name(device), path, "x".join(map(str, shape)), str(batch), schedule, dtype])


def msc_mode(run: int, mode: int) -> int:
    """``mode`` argument of ``critmc_ising_msc_run`` for a rows-per-thread choice."""
    return mode | ((int(run).bit_length()) << 8)


def _time(fn, reps: int, device) -> float:
    """Median device seconds of ``fn`` over ``reps`` calls (after one warm-up)."""
    fn()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize(device)
        out.append(e0.elapsed_time(e1) * 1e-3)
    return float(np.median(out))


def tune_msc(shape, n_chains: int, *, beta: float = 0.4406868, h: float = 0.0, schedule=((0, 1),),
             n_meas: int = 8, device=None, reps: int = 3, force: bool = False) -> dict:
    """Fastest (run, k_inline, mode) of ``critmc_ising_msc_run`` for this shape and batch."""
    dev = require_cuda(device)
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    key = cache_key(dev, "ising-msc", shape, n_chains, ",".join(f"{c}:{r}" for c, r in sched), "u32")
    if not force:
        hit = _load().get(key)
        if hit:
            return hit
    dims = tuple(shape) + (1,) * (3 - len(shape))
    lx, ly, lz = dims
    rows = ly * lz
    words = torch.empty((n_chains, 2, rows, lx // 64), dtype=torch.int32, device=dev)
    keys = np.arange(2 * n_chains, dtype=np.uint32).reshape(n_chains, 2)
    st = stream_handle(dev)
    _lib.call_on(dev, "critmc_ising_msc_init", ptr(words), len(shape), lx, ly, lz, n_chains, ptr(to_dev(keys, dev)),
                 0, st)
    running = torch.empty((n_chains, 2), dtype=torch.int64, device=dev)
    _lib.call_on(dev, "critmc_ising_msc_measure", ptr(words), len(shape), lx, ly, lz, n_chains, ptr(running), st)
    tables = ising_tables(2 * len(shape), beta, h)
    e = torch.empty((n_chains, n_meas), dtype=torch.int64, device=dev)
    m = torch.empty_like(e)
    aux = torch.empty((n_chains, n_meas, 4), dtype=torch.int64, device=dev)
    scratch = empty_bytes(_lib.lib().critmc_ising_msc_scratch_bytes(n_chains, n_meas), dev)
    sweep = [0]
    per_meas = int(sched[:, 1].sum())

    def call(run, k_inline, mode):
        _lib.call_on(dev, "critmc_ising_msc_run", ptr(words), len(shape), lx, ly, lz, n_chains, keys.ctypes.data,
                     tables.ctypes.data, 1, sweep[0], sched.ctypes.data, len(sched), n_meas, ptr(running), ptr(e),
                     ptr(m), ptr(aux), ptr(scratch), msc_mode(run, mode), k_inline, st)
        sweep[0] += per_meas * n_meas

    trials = []
    for mode in MSC_MODES:
        for k_inline in MSC_K_INLINE:
            for run in MSC_RUNS:
                if run > rows:
                    continue
                s = _time(lambda: call(run, k_inline, mode), reps, dev)
                trials.append((s, run, k_inline, mode))
    s, run, k_inline, mode = min(trials)
    n_upd = n_chains * lx * ly * lz * per_meas * n_meas
    best = {"run": run, "k_inline": k_inline, "mode": mode, "seconds": s, "updates_per_ns": n_upd / s / 1e9,
            "trials": len(trials), "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(key, best)
    return best


def ising_tables(z: int, beta: float, h: float) -> np.ndarray:
    """(2, 2, 16) acceptance class tables (Metropolis, heat bath) without building a lattice."""
    import ctypes

    out = np.zeros((2, 2, 16), dtype=np.uint32)
    for slot, algo in enumerate((0, 2)):
        flag = ctypes.c_int32(0)
        _lib.call("critmc_ising_class_table", algo, z, float(beta), float(h), out[slot, 0].ctypes.data,
                  out[slot, 1].ctypes.data, ctypes.byref(flag))
    return out


def _lattice(shape):
    from .lattice import hypercubic

    return hypercubic(tuple(shape))


def tune_on_grid(shape, n: int, *, beta: float = 1.0, schedule=((0, 1),), n_meas: int = 64, device=None,
                 reps: int = 3, force: bool = False) -> dict:
    """Fastest thread blocks per chain of the O(n) multi-block lane for one chain."""
    dev = require_cuda(device)
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    key = cache_key(dev, f"on{n}-grid", shape, 1, ",".join(f"{c}:{r}" for c, r in sched), "f32")
    if not force:
        hit = _load().get(key)
        if hit:
            return hit
    from .models import ON
    from .on_models import ONChain

    model = ON(_lattice(shape), n)
    rng = np.random.default_rng(1)
    chain = ONChain(model, model.initial_state("random", rng), np.array([1, 2], dtype=np.uint32), dev,
                    lane="grid")
    slots = int(np.prod(shape)) // 2
    cands = sorted({max(1, -(-slots // (256 * f))) for f in (1, 2, 4, 8, 16)})
    trials = []
    for blocks in cands:
        chain.blocks_per_chain = blocks
        s = _time(lambda: chain.advance({"step": 1.0}, beta, sched, n_meas), reps, dev)
        trials.append((s, blocks))
    s, blocks = min(trials)
    best = {"blocks_per_chain": blocks, "seconds_per_meas": s / n_meas, "trials": len(trials),
            "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(key, best)
    return best


# representative (lane, family) -> (request kind, sizes) measured for the serving cost model
_SERVE_PROBES = {
    ("items", "byte"): ("ising", (16, 32)),
    ("items", "msc"): ("ising", (64, 256)),
    ("items", "potts"): ("potts", (32, 128)),
    ("items", "on2"): ("xy", (32, 128)),
    ("items", "on3"): ("heisenberg", (16, 64)),
    ("grid", "msc"): ("ising", (512, 1024)),
    ("grid", "on2"): ("xy", (64, 128)),
    ("grid", "on3"): ("heisenberg", (64, 128)),
}
# teams: (lane, family) -> probe, for every team size
_TEAM_PROBES = {"msc": ("ising", (256, 1024)), "byte": ("ising", (32, 128)), "potts": ("potts", (64, 128)),
                "on2": ("xy", (64, 128)), "on3": ("heisenberg", (32, 64))}
for _t in (2, 4, 8, 16):
    for _fam, _probe in _TEAM_PROBES.items():
        _SERVE_PROBES[(f"team{_t}", _fam)] = _probe


def calibrate_serving(device=None, *, n_meas: int = 200, force: bool = False) -> dict:
    """Per-lane cost model (a, b): seconds per sweep = a + b * sites, from two sizes each."""
    dev = require_cuda(device)
    key = cache_key(dev, "serve-costs", (1,), 1, "metropolis", "mixed")  # (1,): with team lanes
    if not force:
        hit = _load().get(key)
        if hit:
            return {tuple(k.split("/")): tuple(v) for k, v in hit["costs"].items()}
    from .items import ItemRun, run_items
    from .serve import Request, open_chain

    costs = {}
    for (lane, family), (kind, sizes) in _SERVE_PROBES.items():
        pts = []
        for L in sizes:
            req = Request(kind, L, 0.44 if kind == "ising" else (1.4 if kind == "potts" else 1.1), n_meas)
            model, chain, running = open_chain(req, dev)
            sched = req.schedule()
            if lane == "items" or lane.startswith("team"):
                team = int(lane[4:]) if lane.startswith("team") else 1

                def fn():
                    run_items([ItemRun(model, chain, running, req.beta, sched, n_meas, team=team)], dev)
            else:
                if hasattr(chain, "lane"):
                    chain.lane = "grid"

                def fn():
                    model.advance(chain, running, req.beta, sched, n_meas)
            pts.append((req.n_sites, _time(fn, 3, dev) / n_meas))
        (n0, t0), (n1, t1) = pts
        b = max(0.0, (t1 - t0) / (n1 - n0))
        a = max(1e-7, t0 - b * n0)
        costs[(lane, family)] = (a, b)
    _store(key, {"costs": {f"{k[0]}/{k[1]}": list(v) for k, v in costs.items()},
                 "when": time.strftime("%Y-%m-%dT%H:%M:%S")})
    return costs
