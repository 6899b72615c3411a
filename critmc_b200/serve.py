"""Serving: simulation requests of mixed models and sizes, continuously batched.

A ``Server`` admits ``Request`` objects (model, lattice size, beta, number of
measured sweeps, seed) in arrival order while their lattices fit in the HBM
budget, keeps each admitted request's lattice, running sums and sweep counter
resident on the device, and advances all admitted requests together in ticks:

* lattices that fit in shared memory run as work items of the persistent
  per-family kernels (``critmc_run_items``: one thread block per chain,
  blocks pull chains from a queue, the three family kernels side by side);
* large multi-spin-coded Ising lattices run on the multi-block half-sweep
  kernel (``critmc_ising_msc_run``), one library stream per request, next to
  the item kernels.

Each tick gives every request a slice of sweeps sized so the tick takes about
``tick_ms`` of GPU time; requests that arrive meanwhile are admitted at the
next tick, so new work joins the running batch instead of waiting for it to
drain.  Two ticks are in flight: the host plans and launches tick k+1 while
tick k's measurements come back.  Every random number is a function of the
request's Philox key, its sweep index and the site, so a request's series are
the same alone and in any mix (``open_chain`` + ``Model.advance`` reproduce
them one request at a time).

critmc has no serving layer; its batch runner (src/critmc/runner.py:154-223)
runs one chain per CPU process.
"""

from __future__ import annotations

import ctypes
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .device import empty_bytes, ptr, require_cuda
from .items import ITEM_BYTE_ISING, ITEM_MSC_ISING, ITEM_ON, ITEM_POTTS, CritmcItem, launch_items
from .lattice import hypercubic
from .models import ON, UPDATE_CODES, Ising, Model, Potts, _IsingMscChain, _msc_ok
from .rng import make_rng, philox_key
from .sim import parse_updates

__all__ = ["Request", "Result", "Server", "open_chain", "mixed_workload", "DEFAULT_UPDATES"]

DEFAULT_UPDATES = {"ising": "metropolis", "potts": "metropolis", "xy": "heatbath", "heisenberg": "heatbath"}

_I8, _F8 = np.dtype(np.int64), np.dtype(np.float64)
_ALIGN = 256
GRID_MAX_MEAS = 4096  # measurements per grid-lane call (bounds its scratch)

# Seconds per sweep of one chain, a + b * sites, by (lane, family): starting
# values for the tick planner (B200 measurements of one chain alone); the
# planner rescales them from the measured tick times.
COSTS = {
    ("items", "msc"): (2.7e-6, 5.0e-11),
    ("items", "byte"): (2.0e-6, 5.0e-10),
    ("items", "potts"): (1.9e-6, 1.0e-9),
    ("items", "on2"): (5.0e-6, 5.5e-9),
    ("items", "on3"): (6.0e-6, 8.0e-9),
    ("grid", "msc"): (8.7e-6, 2.0e-13),
    ("grid", "on2"): (1.0e-5, 2.0e-10),
    ("grid", "on3"): (1.2e-5, 3.0e-10),
}


@dataclass
class Request:
    """One simulation request: ``sweeps`` applications of ``updates``, one measurement each."""

    model: str  # "ising", "potts", "xy", "heisenberg"
    L: int
    beta: float
    sweeps: int
    seed: int = 0
    dim: int = 2
    q: int = 10
    h: float = 0.0
    updates: str | None = None
    rid: int = -1
    arrival: float | None = None  # seconds after the server's start; None = when submitted

    @property
    def shape(self) -> tuple[int, ...]:
        return (int(self.L),) * int(self.dim)

    @property
    def n_sites(self) -> int:
        return int(self.L) ** int(self.dim)

    def schedule(self) -> np.ndarray:
        rows = parse_updates(self.updates or DEFAULT_UPDATES[self.model])
        return np.array([[UPDATE_CODES[n], 1 if k is None else k] for n, k in rows], dtype=np.int64)


@dataclass
class Result:
    request: Request
    series: dict[str, np.ndarray]  # full series, or column sums (``summary`` servers)
    state: np.ndarray | None
    arrival: float
    admitted: float
    finished: float
    updates: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def build_model(req: Request, cache: dict | None = None) -> Model:
    key = (req.model, req.dim, req.L, req.q, req.h)
    if cache is not None and key in cache:
        return cache[key]
    lat = hypercubic(req.shape)
    if req.model == "ising":
        m = Ising(lat, req.h)
    elif req.model == "potts":
        m = Potts(lat, req.q)
    elif req.model in ("xy", "heisenberg"):
        m = ON(lat, 2 if req.model == "xy" else 3)
    else:
        raise ValueError(f"unknown model {req.model!r}")
    if cache is not None:
        cache[key] = m
    return m


def open_chain(req: Request, device=None, cache: dict | None = None):
    """``(model, chain, running)`` of a request's random start on ``device``.

    The Philox key comes from ``make_rng(seed, "request", model, L)``;
    multi-spin-coded Ising lattices are drawn on the device, the others on
    the host.  ``model.advance(chain, running, beta, schedule, n)`` then gives
    the request's series as the server does.
    """
    model = build_model(req, cache)
    model.check_updates([n for n, _ in parse_updates(req.updates or DEFAULT_UPDATES[req.model])])
    rng = make_rng(req.seed, "request", req.model, req.L)
    if isinstance(model, Ising) and _msc_ok(req.shape):
        chain = _IsingMscChain.on_device(model, philox_key(rng), device)
        eb, m = (int(v) for v in chain.measure().cpu().numpy().ravel())
        return model, chain, {"e_b": eb, "m": m}
    state = model.initial_state("random", rng)
    chain = model.to_device(state, rng, device)
    return model, chain, model.begin(state)


def mixed_workload(n: int, rate: float, seed: int = 0) -> list[Request]:
    """Seeded Poisson stream of mixed requests.

    Each request is, with probability 1/3 each: 2D Ising with L in
    {16, ..., 1024} and beta ~ U[0.38, 0.50]; q=10 Potts with L in
    {16, ..., 128} and beta ~ U[1.35, 1.50]; XY with L in {32, 64, 128} and
    T ~ U[0.8, 1.0].  Sweeps are log-uniform in [1e3, 1e5]; arrival gaps are
    exponential with mean 1/rate.
    """
    rng = make_rng(seed, "serve-workload")
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    kinds = rng.integers(0, 3, n)
    u = rng.random(n)
    sizes = rng.integers(0, 1 << 30, n)
    sweeps = np.rint(10.0 ** rng.uniform(3.0, 5.0, n)).astype(np.int64)
    out = []
    for i in range(n):
        if kinds[i] == 0:
            L = (16, 32, 64, 128, 256, 512, 1024)[sizes[i] % 7]
            r = Request("ising", L, 0.38 + 0.12 * u[i], int(sweeps[i]))
        elif kinds[i] == 1:
            L = (16, 32, 64, 128)[sizes[i] % 4]
            r = Request("potts", L, 1.35 + 0.15 * u[i], int(sweeps[i]), q=10)
        else:
            L = (32, 64, 128)[sizes[i] % 3]
            r = Request("xy", L, 1.0 / (0.8 + 0.2 * u[i]), int(sweeps[i]))
        r.seed, r.rid, r.arrival = seed * 1_000_003 + i, i, float(arrivals[i])
        out.append(r)
    return out


@dataclass
class _Job:
    req: Request
    model: Model
    chain: object
    running: dict
    lane: str  # "items" or "grid"
    family: str
    sched: np.ndarray
    sweeps_per_meas: int
    fields: list  # (name, dtype, width)
    item: CritmcItem | None
    tensors: dict
    dev_bytes: int
    admitted: float
    series: dict = field(default_factory=dict)
    tables: object = None  # host tables of the multi-block lane
    launched: int = 0
    harvested: int = 0

    @property
    def meas_bytes(self) -> int:
        return sum(8 * w for _, _, w in self.fields)


@dataclass
class _Tick:
    slot: int
    entries: list  # (job, n_meas, offset)
    used: int
    predicted: float
    start: torch.cuda.Event
    end: torch.cuda.Event
    done: torch.cuda.Event


class Server:
    """Continuous-batching sampler for a stream of mixed requests on one GPU."""

    def __init__(self, device=None, *, hbm_budget: int | None = None, reserve: int = 1 << 30,
                 tick_ms: float = 20.0, max_active: int = 4096, grid_min_sites: int = 1 << 18,
                 arena_bytes: int = 64 << 20, keep_series: bool = True, keep_state: bool = False,
                 grid_streams: int = 16, on_result=None):
        self.device = require_cuda(device)
        free, _ = torch.cuda.mem_get_info(self.device)
        cap = max(0, free - reserve)
        self.budget = min(cap, int(hbm_budget)) if hbm_budget is not None else cap
        self.tick_s = tick_ms * 1e-3
        self.max_active = max_active
        self.grid_min_sites = grid_min_sites
        self.keep_series, self.keep_state = keep_series, keep_state
        self.on_result = on_result
        self.in_use = 0
        self.peak_in_use = 0
        self.queue: deque[Request] = deque()
        self.active: list[_Job] = []
        self.results: list[Result] = []
        self.inflight: deque[_Tick] = deque()
        self.models: dict = {}
        self.stream = torch.cuda.Stream(self.device)
        self.admit_stream = torch.cuda.Stream(self.device)
        self.grid_pool = [torch.cuda.Stream(self.device) for _ in range(grid_streams)]
        self.arena_bytes = int(arena_bytes)
        self.arena = [empty_bytes(self.arena_bytes, self.device) for _ in range(2)]
        self.host = [torch.empty(self.arena_bytes, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        self.staging = [None, None]
        # sized once: a buffer replaced while a tick still reads it would be recycled too early
        self.item_buffer = empty_bytes(_lib.lib().critmc_items_buffer_bytes(max_active), self.device)
        self.grid_scratch = [None] * grid_streams
        self.scale = 1.0
        self.costs = dict(COSTS)
        self.ticks = 0
        self.gpu_seconds = 0.0
        self.updates_done = 0
        self.max_queued = 0
        self._next_rid = 0
        self.t0 = time.perf_counter()

    # ---- bookkeeping ---------------------------------------------------
    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, req: Request) -> Request:
        if req.rid < 0:
            req.rid = self._next_rid
        self._next_rid = max(self._next_rid, req.rid + 1)
        if req.arrival is None:
            req.arrival = self.now()
        if self.queue and req.arrival < self.queue[-1].arrival:
            raise ValueError("requests must be submitted in arrival order")
        self.queue.append(req)
        return req

    @staticmethod
    def request_bytes(req: Request) -> int:
        """Device bytes a request holds while admitted (lattice + running sums)."""
        n = req.n_sites
        if req.model == "ising":
            lat = n // 8 if _msc_ok(req.shape) else n
        elif req.model == "potts":
            lat = n + 8 * req.q
        else:
            lat = 4 * n * (2 if req.model == "xy" else 3)
        return lat + 4096

    # ---- admission -------------------------------------------------------
    def _admit(self) -> None:
        admitted = False
        now = self.now()
        while self.queue and self.queue[0].arrival <= now and len(self.active) < self.max_active:
            req = self.queue[0]
            need = self.request_bytes(req)
            if need > self.budget:
                raise ValueError(f"request {req.rid} needs {need} device bytes, above the budget {self.budget}")
            if self.in_use + need > self.budget:
                break
            self.queue.popleft()
            with torch.cuda.stream(self.admit_stream):
                job = self._open(req, need)
            self.in_use += need
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            self.active.append(job)
            admitted = True
        waiting = 0
        for r in self.queue:
            if r.arrival > now:
                break
            waiting += 1
        self.max_queued = max(self.max_queued, waiting)
        if admitted:
            ev = torch.cuda.Event()
            ev.record(self.admit_stream)
            self.stream.wait_event(ev)

    def _open(self, req: Request, need: int) -> _Job:
        model, chain, running = open_chain(req, self.device, self.models)
        sched = req.schedule()
        dev = self.device
        t: dict = {}
        item = None
        tables = None
        dim = len(req.shape)
        if isinstance(model, Ising):
            msc = isinstance(chain, _IsingMscChain)
            family = "msc" if msc else "byte"
            fields = [("Eb", _I8, 1), ("M", _I8, 1), ("aux", _I8, 4)]
            t["running"] = torch.tensor([[running["e_b"], running["m"]]], dtype=torch.int64, device=dev)
            lane = "grid" if msc and req.n_sites >= self.grid_min_sites else "items"
            kind = ITEM_MSC_ISING if msc else ITEM_BYTE_ISING
            h = model.h
            if lane == "grid":
                tables = np.ascontiguousarray(model.tables(req.beta)[0])
        elif isinstance(model, Potts):
            family, lane, kind, h = "potts", "items", ITEM_POTTS, 0.0
            fields = [("E", _I8, 1), ("counts", _I8, model.q), ("aux", _I8, 4)]
            t["running"] = torch.tensor([running["energy"]], dtype=torch.int64, device=dev)
            t["counts"] = torch.from_numpy(np.asarray(running["counts"], dtype=np.int64)).to(dev)
        else:
            family, lane, kind, h = f"on{model.n}", chain.lane.replace("block", "items"), ITEM_ON, 0.0
            fields = [("E", _F8, 1), ("M", _F8, model.n), ("stiff_c", _F8, dim), ("stiff_s", _F8, dim),
                      ("aux", _I8, 4)]
            tables = (np.array([req.beta], dtype=np.float64),
                      np.array([running.get("step", 1.0)], dtype=np.float64))
        if lane == "items":
            item = CritmcItem()
            item.spins = ptr(chain.words if family == "msc" else chain.spins)
            item.kind = kind
            item.dim = dim
            item.lx, item.ly, item.lz = chain.dims
            item.q_or_n = model.q if family == "potts" else (model.n if kind == ITEM_ON else 0)
            item.key[0], item.key[1] = int(chain.key.ravel()[0]), int(chain.key.ravel()[1])
            if len(sched) > 4:
                raise ValueError("served schedules have at most 4 rows")
            item.n_rows = len(sched)
            for r, (code, reps) in enumerate(sched):
                item.codes[r], item.reps[r] = int(code), int(reps)
            item.running = ptr(t.get("running"))
            item.counts = ptr(t.get("counts"))
            _lib.call("critmc_item_prepare", ctypes.byref(item), float(req.beta), float(h),
                      float(running.get("step", 1.0)))
        job = _Job(req, model, chain, running, lane, family, sched, int(sched[:, 1].sum()), fields, item, t,
                   need, self.now(), tables=tables)
        if self.keep_series:
            job.series = {name: np.empty((req.sweeps, w) if w > 1 else req.sweeps, dtype=dt)
                          for name, dt, w in fields}
        else:
            job.series = {name: np.zeros(w, dtype=dt) for name, dt, w in fields}
        return job

    # ---- ticks -----------------------------------------------------------
    def _sweep_seconds(self, job: _Job) -> float:
        a, b = self.costs[(job.lane, job.family)]
        return job.sweeps_per_meas * (a + b * job.req.n_sites)

    def _plan(self):
        jobs = [j for j in self.active if j.launched < j.req.sweeps]
        if not jobs:
            return [], 0.0
        plan = []
        n_grid = sum(1 for j in jobs if j.lane == "grid")
        share = max(1, -(-n_grid // len(self.grid_pool)))  # grid jobs per library stream
        for j in jobs:
            per = self._sweep_seconds(j) * self.scale
            target = self.tick_s / share if j.lane == "grid" else self.tick_s
            n = max(1, int(target / per))
            n = min(n, j.req.sweeps - j.launched)
            if j.lane == "grid":
                n = min(n, GRID_MAX_MEAS)
            plan.append([j, n])
        total = sum(_round_up(j.meas_bytes * n) for j, n in plan)
        if total > self.arena_bytes:
            f = self.arena_bytes / total
            for p in plan:
                p[1] = max(1, int(p[1] * f * 0.98))
            while sum(_round_up(j.meas_bytes * n) for j, n in plan) > self.arena_bytes and len(plan) > 1:
                plan.pop()
        item_t = [self._sweep_seconds(j) * self.scale * n for j, n in plan if j.lane == "items"]
        grid_t = sorted((self._sweep_seconds(j) * self.scale * n for j, n in plan if j.lane == "grid"),
                        reverse=True)
        loads = [0.0] * len(self.grid_pool)
        for t in grid_t:  # the launch assigns grid jobs longest first to the least loaded stream
            loads[loads.index(min(loads))] += t
        predicted = max(item_t + loads)
        return plan, predicted

    def _launch(self, plan, predicted) -> _Tick:
        slot = self.ticks % 2
        self.ticks += 1
        base = ptr(self.arena[slot])
        entries = []
        off = 0
        items = []
        grid = []
        for j, n in plan:
            entries.append((j, n, off))
            ptrs = []
            o = off
            for _, _, w in j.fields:
                ptrs.append(base + o)
                o += 8 * w * n
            if j.lane == "items":
                it = CritmcItem.from_buffer_copy(j.item)
                it.sweep0 = j.chain.sweep
                it.n_meas = n
                it.e_out, it.vec_out, it.aux_out = ptrs[0], ptrs[1], ptrs[-1]
                if j.family.startswith("on"):
                    it.sc_out, it.ss_out = ptrs[2], ptrs[3]
                items.append(it)
            else:
                grid.append((j, n, ptrs))
            off = _round_up(off + j.meas_bytes * n)
        s = self.stream
        start, end, done = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
                            torch.cuda.Event())
        start.record(s)
        if items:
            need = len(items) * ctypes.sizeof(CritmcItem)
            if self.staging[slot] is None or self.staging[slot].numel() < need:
                self.staging[slot] = torch.empty(max(need, 1 << 16), dtype=torch.uint8, pin_memory=True)
            arr = (CritmcItem * len(items))(*items)
            self.item_buffer = launch_items(arr, self.device, self.item_buffer, staging=self.staging[slot],
                                            stream=s.cuda_stream)
        if grid:
            fork = torch.cuda.Event()
            fork.record(s)
            used = set()
            loads = [0.0] * len(self.grid_pool)
            grid.sort(key=lambda g: -self._sweep_seconds(g[0]) * g[1])
            for j, n, ptrs in grid:
                k = loads.index(min(loads))
                loads[k] += self._sweep_seconds(j) * n
                gs = self.grid_pool[k]
                if k not in used:
                    gs.wait_event(fork)
                    used.add(k)
                scratch = self._grid_scratch(k)
                c = j.chain
                lx, ly, lz = c.dims
                if j.family == "msc":
                    _lib.call("critmc_ising_msc_run", ptr(c.words), len(c.shape), lx, ly, lz, 1,
                              c.key.ctypes.data, j.tables.ctypes.data, 1, c.sweep, j.sched.ctypes.data,
                              len(j.sched), n, ptr(j.tensors["running"]), ptrs[0], ptrs[1], ptrs[2],
                              ptr(scratch), 0, c.k_inline, gs.cuda_stream)
                else:
                    betas, steps = j.tables
                    _lib.call("critmc_on_run_grid", ptr(c.spins), len(c.shape), lx, ly, lz, c.n, 1,
                              c.key.ctypes.data, betas.ctypes.data, steps.ctypes.data, 1, c.sweep,
                              j.sched.ctypes.data, len(j.sched), n, ptrs[0], ptrs[1], ptrs[2], ptrs[3],
                              ptrs[4], ptr(scratch), c.blocks_per_chain, gs.cuda_stream)
            for k in used:
                join = torch.cuda.Event()
                join.record(self.grid_pool[k])
                s.wait_event(join)
        end.record(s)
        with torch.cuda.stream(s):
            if off:
                self.host[slot][:off].copy_(self.arena[slot][:off], non_blocking=True)
        done.record(s)
        for j, n, _ in entries:
            j.launched += n
            j.chain.sweep += n * j.sweeps_per_meas
        return _Tick(slot, entries, off, predicted, start, end, done)

    def _grid_scratch(self, k: int) -> torch.Tensor:
        if self.grid_scratch[k] is None:
            lib = _lib.lib()
            need = max(lib.critmc_ising_msc_scratch_bytes(1, GRID_MAX_MEAS),
                       lib.critmc_on_grid_scratch_bytes(1, GRID_MAX_MEAS, 3, 3))
            self.grid_scratch[k] = empty_bytes(need, self.device)
        return self.grid_scratch[k]

    def _harvest(self, tick: _Tick) -> None:
        tick.done.synchronize()
        gpu = tick.start.elapsed_time(tick.end) * 1e-3
        self.gpu_seconds += gpu
        if tick.predicted > 0 and gpu > 0:
            # damped correction of the tick planner's cost model
            self.scale *= min(4.0, max(0.25, (gpu / tick.predicted))) ** 0.5
        host = self.host[tick.slot].numpy()
        now = self.now()
        for j, n, off in tick.entries:
            o = off
            h0 = j.harvested
            for name, dt, w in j.fields:
                cnt = n * w
                v = np.frombuffer(host, dtype=dt, count=cnt, offset=o)
                o += 8 * cnt
                if self.keep_series:
                    j.series[name][h0:h0 + n] = v.reshape(n, w) if w > 1 else v
                else:
                    j.series[name] += v.reshape(n, w).sum(axis=0)
            j.harvested += n
            self.updates_done += n * j.sweeps_per_meas * j.req.n_sites
            if j.harvested == j.req.sweeps:
                self._finish(j, now)

    def _finish(self, j: _Job, now: float) -> None:
        req = j.req
        if "running" in j.tensors:
            r = j.tensors["running"].cpu().numpy().ravel()
            if isinstance(j.model, Ising):
                j.running["e_b"], j.running["m"] = int(r[0]), int(r[1])
            else:
                j.running["energy"] = int(r[0])
                j.running["counts"] = j.tensors["counts"].cpu().numpy().copy()
        series = j.series
        if isinstance(j.model, Ising) and self.keep_series:
            series["E"] = series["Eb"] - j.model.h * series["M"] if j.model.h != 0.0 else series["Eb"]
        state = j.chain.fetch() if self.keep_state else None
        res = Result(req, series, state, float(req.arrival), j.admitted, now,
                     req.n_sites * j.sweeps_per_meas * req.sweeps)
        self.active.remove(j)
        self.in_use -= j.dev_bytes
        j.chain = None
        j.tensors.clear()
        if self.on_result is not None:
            self.on_result(res)
        else:
            self.results.append(res)

    # ---- driving ---------------------------------------------------------
    def step(self) -> bool:
        """Admit, launch one tick, harvest the older tick; False when idle."""
        self._admit()
        plan, predicted = self._plan()
        if plan:
            self.inflight.append(self._launch(plan, predicted))
        if self.inflight and (len(self.inflight) >= 2 or not plan):
            self._harvest(self.inflight.popleft())
        return bool(self.queue or self.active or self.inflight)

    def run(self, requests=None) -> list[Result]:
        """Submit ``requests`` (in arrival order) and serve until all are done."""
        for r in requests or ():
            self.submit(r)
        while self.step():
            if not self.active and not self.inflight and self.queue:
                wait = self.queue[0].arrival - self.now()
                if wait > 0:
                    time.sleep(wait)
        return self.results

    def stats(self) -> dict:
        return {"ticks": self.ticks, "gpu_seconds": self.gpu_seconds, "updates": self.updates_done,
                "peak_hbm_bytes": self.peak_in_use, "hbm_budget": self.budget,
                "max_queued": self.max_queued}


def _round_up(n: int) -> int:
    return (n + _ALIGN - 1) // _ALIGN * _ALIGN

