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
from .on_models import GRID_MIN_SITES as ON_GRID_MIN_SITES
from .rng import make_rng, philox_key
from .sim import parse_updates
from .streaming import HostStreamStats

__all__ = ["Request", "Result", "Server", "open_chain", "mixed_workload", "DEFAULT_UPDATES"]

# critmc's Simulation default (src/critmc/sim.py:157) for every model
DEFAULT_UPDATES = {"ising": "metropolis", "potts": "metropolis", "xy": "metropolis", "heisenberg": "metropolis"}

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
    ("items", "on2"): (3.0e-6, 2.5e-9),
    ("items", "on3"): (4.0e-6, 4.0e-9),
    ("grid", "msc"): (8.7e-6, 2.0e-13),
    ("grid", "on2"): (1.0e-5, 2.0e-10),
    ("grid", "on3"): (1.2e-5, 3.0e-10),
}
TEAMS = (2, 4, 8, 16)
# teams (thread-block clusters per item), measured on B200 for T = 2..16: about
# 1/T of one block's per-site time, and 2-3 times its fixed time per sweep
# (cluster barriers, the lattice in global memory)
for _fam in ("msc", "byte", "potts", "on2", "on3"):
    _a, _b = COSTS[("items", _fam)]
    for _t in TEAMS:
        COSTS[(f"team{_t}", _fam)] = (2.5 * _a, 1.1 * _b / _t)
TEAM_SLACK = 1.15  # a smaller team within this factor of the fastest saves SMs


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
    stats: dict | None = None  # summary servers: Gamma-method mean, error, tau_int per scalar series

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
    group: str = ""
    team: int = 1  # thread blocks per item on an item lane
    home: object = None  # the lane that advances it
    stream: dict = field(default_factory=dict)  # summary mode: streaming statistics per scalar field

    @property
    def meas_bytes(self) -> int:
        return sum(8 * w for _, _, w in self.fields)


@dataclass
class _Tick:
    lane: "_Lane"
    entries: list  # (job, n_meas, offset)
    offset: int  # arena segment
    size: int
    predicted: float
    start: torch.cuda.Event
    end: torch.cuda.Event
    done: torch.cuda.Event
    seq: int = 0


class _Lane:
    """Jobs advanced by one launch sequence per tick on one stream.

    An item lane holds the requests of one persistent-kernel group (their
    ticks are one ``critmc_run_items`` call); a grid lane holds one request
    on the multi-block kernels.  Lanes tick independently, two ticks in
    flight each, so a lane of short sweeps never waits for a lane of long ones.
    """

    def __init__(self, kind: str, family: str, stream: torch.cuda.Stream):
        self.kind, self.family, self.stream = kind, family, stream
        self.jobs: list[_Job] = []
        self.inflight: deque[_Tick] = deque()
        self.scale = 1.0
        self.staging = [None, None]
        self.n_ticks = 0
        self.item_buffer = None


class _Arena:
    """First-fit allocator of tick output segments in a device/pinned-host pair."""

    def __init__(self, size: int, device):
        self.size = size
        self.dev = empty_bytes(size, device)
        self.host = torch.empty(size, dtype=torch.uint8, pin_memory=True)
        self.host_np = self.host.numpy()
        self.free = [(0, size)]

    def alloc(self, n: int) -> int | None:
        n = _round_up(max(n, 1))
        for i, (o, sz) in enumerate(self.free):
            if sz >= n:
                if sz == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (o + n, sz - n)
                return o
        return None

    def release(self, o: int, n: int) -> None:
        n = _round_up(max(n, 1))
        self.free.append((o, n))
        self.free.sort()
        merged = []
        for a, sz in self.free:
            if merged and merged[-1][0] + merged[-1][1] == a:
                merged[-1] = (merged[-1][0], merged[-1][1] + sz)
            else:
                merged.append((a, sz))
        self.free = merged


class Server:
    """Continuous-batching sampler for a stream of mixed requests on one GPU."""

    def __init__(self, device=None, *, hbm_budget: int | None = None, reserve: int = 1 << 30,
                 tick_ms: float = 10.0, max_active: int = 4096, grid_min_sites: int = 1 << 18,
                 grid_after_s: float | None = None, team_after_s: float | None = 1.0, max_team: int = 8,
                 max_grid_lanes: int = 8, arena_bytes: int = 256 << 20, keep_series: bool = True,
                 keep_state: bool = False, grid_streams: int = 32, on_result=None, costs=None,
                 stats_lag: int = 64):
        self.device = require_cuda(device)
        free, _ = torch.cuda.mem_get_info(self.device)
        cap = max(0, free - reserve - 2 * arena_bytes)
        self.budget = min(cap, int(hbm_budget)) if hbm_budget is not None else cap
        self.tick_s = tick_ms * 1e-3
        self.max_active = max_active
        self.grid_min_sites = grid_min_sites
        # None: multi-block lanes for multi-spin-coded Ising lattices from grid_min_sites
        # sites and O(n) lattices from 4096 sites, first come first served; a number:
        # for the requests that an item lane would keep longer than that (cost model)
        self.grid_after_s = grid_after_s
        # the multi-block lanes are launch-bound: they buy latency, the item
        # kernels throughput, so at most this many requests use them at once
        self.max_grid_lanes = max_grid_lanes
        # None: one block per item.  A number: a request that one block would
        # keep longer than that (cost model) gets a team, the smallest thread-
        # block cluster predicted to finish it within that time (else the
        # fastest); teams replace the multi-block lanes for the families they
        # serve.  Teams of at most max_team blocks: on the 10,000-request mix,
        # 1 s with teams of up to 8 or 16 gave p99 1.1 s (one block per item:
        # 5.1 s); 0.5 s with up to 16 blocks gave 5.2 s once (16-block clusters
        # waiting for 16 free SMs of one GPC), with up to 8 blocks 1.1 s
        self.team_after_s = team_after_s
        self.teams = tuple(t for t in TEAMS if t <= max_team)
        self._team_ok: dict = {}
        self.team_sizes_used: set[int] = set()
        self.keep_series, self.keep_state = keep_series, keep_state
        self.stats_lag = int(stats_lag)
        self.on_result = on_result
        self.in_use = 0
        self.peak_in_use = 0
        self.queue: deque[Request] = deque()
        self.active: list[_Job] = []
        self.results: list[Result] = []
        self.models: dict = {}
        self.admit_stream = torch.cuda.Stream(self.device)
        self.admit_event: torch.cuda.Event | None = None
        self.item_lanes: dict[str, _Lane] = {}
        self.grid_pool = [torch.cuda.Stream(self.device) for _ in range(grid_streams)]
        self.grid_lanes: list[_Lane] = []
        self._next_grid = 0
        self.arena = _Arena(int(arena_bytes), self.device)
        self.grid_scratch: dict[int, torch.Tensor] = {}
        self.costs = dict(COSTS)
        if costs == "auto":  # the autotuner's measured cost model (cached per GPU)
            from .autotune import calibrate_serving

            self.costs.update(calibrate_serving(self.device))
        elif costs is not None:
            self.costs.update(costs)
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

    def _wants_grid(self, req: Request, family: str) -> bool:
        """Multi-block lanes are few (launch-bound); they go to the requests that an
        item lane would keep longest: at least grid_min_sites sites and, by the
        cost model, more than grid_after_s seconds of item-lane time."""
        if self.grid_after_s is None:
            return req.n_sites >= (self.grid_min_sites if family == "msc" else ON_GRID_MIN_SITES)
        if req.n_sites < ON_GRID_MIN_SITES:
            return False
        a, b = self.costs[("items", family)]
        per_meas = int(req.schedule()[:, 1].sum())
        return req.sweeps * per_meas * (a + b * req.n_sites) > self.grid_after_s

    def _team_for(self, req: Request, family: str) -> int:
        """Blocks per item for a request on an item lane (1 = one block): the
        smallest team predicted to finish within team_after_s; else the smallest
        team within TEAM_SLACK of the fastest (larger teams buy little there and
        hold more SMs)."""
        if self.team_after_s is None:
            return 1
        per = req.sweeps * int(req.schedule()[:, 1].sum())
        a, b = self.costs[("items", family)]
        pred = {1: per * (a + b * req.n_sites)}
        if pred[1] <= self.team_after_s:
            return 1
        for t in self.teams:
            if not self._team_fits(req, family, t):
                continue
            a, b = self.costs[(f"team{t}", family)]
            pred[t] = per * (a + b * req.n_sites)
            if pred[t] <= self.team_after_s:
                return t
        fastest = min(pred.values())
        return min(t for t, p in pred.items() if p <= TEAM_SLACK * fastest)

    def _team_fits(self, req: Request, family: str, team: int) -> bool:
        """Whether this GPU schedules teams of that size for the request's kernel
        (asked once per kernel and size)."""
        kind = {"msc": ITEM_MSC_ISING, "byte": ITEM_BYTE_ISING, "potts": ITEM_POTTS}.get(family, ITEM_ON)
        n = int(family[2:]) if family.startswith("on") else 0
        key = (kind, n, len(req.shape), team)
        if key not in self._team_ok:
            from .items import team_clusters

            self._team_ok[key] = team_clusters(kind, n, len(req.shape), team, self.device) > 0
        return self._team_ok[key]

    def _grid_free(self) -> bool:
        return sum(1 for lane in self.grid_lanes if lane.jobs) < self.max_grid_lanes

    def _lanes(self):
        yield from self.item_lanes.values()
        yield from self.grid_lanes

    # ---- admission -------------------------------------------------------
    def _admit(self) -> bool:
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
            self._assign(job)
            admitted = True
        waiting = 0
        for r in self.queue:
            if r.arrival > now:
                break
            waiting += 1
        self.max_queued = max(self.max_queued, waiting)
        if admitted:
            self.admit_event = torch.cuda.Event()
            self.admit_event.record(self.admit_stream)
        return admitted

    def _assign(self, job: _Job) -> None:
        if job.lane == "items":
            key = job.group
            lane = self.item_lanes.get(key)
            if lane is None:
                lane = self.item_lanes[key] = _Lane("items", job.family, torch.cuda.Stream(self.device))
        else:
            stream = self.grid_pool[self._next_grid % len(self.grid_pool)]
            self._next_grid += 1
            lane = _Lane("grid", job.family, stream)
            self.grid_lanes.append(lane)
        lane.jobs.append(job)
        job.home = lane

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
            group = family
            fields = [("Eb", _I8, 1), ("M", _I8, 1), ("aux", _I8, 4)]
            t["running"] = torch.tensor([[running["e_b"], running["m"]]], dtype=torch.int64, device=dev)
            team = self._team_for(req, family)
            if self.team_after_s is not None:
                lane = "items" if (team > 1 or not msc or req.n_sites <= 1 << 20) else "grid"
            else:
                lane = "grid" if msc and self._wants_grid(req, "msc") and self._grid_free() else "items"
            kind = ITEM_MSC_ISING if msc else ITEM_BYTE_ISING
            h = model.h
            if lane == "grid":
                tables = np.ascontiguousarray(model.tables(req.beta)[0])
        elif isinstance(model, Potts):
            family, group, lane, kind, h = "potts", "byte", "items", ITEM_POTTS, 0.0
            team = self._team_for(req, family)
            fields = [("E", _I8, 1), ("counts", _I8, model.q), ("aux", _I8, 4)]
            t["running"] = torch.tensor([running["energy"]], dtype=torch.int64, device=dev)
            t["counts"] = torch.from_numpy(np.asarray(running["counts"], dtype=np.int64)).to(dev)
        else:
            # same results on either lane
            team = self._team_for(req, f"on{model.n}")
            grid = self.team_after_s is None and self._wants_grid(req, f"on{model.n}") and self._grid_free()
            chain.lane = "grid" if grid else "block"
            family, lane, kind, h = f"on{model.n}", chain.lane.replace("block", "items"), ITEM_ON, 0.0
            group = f"on{model.n}d{dim}"
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
            item.team = team
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
        # item lanes by kernel group, team size and lattice size class (a call's blocks get
        # the largest lattice's shared memory, so small lattices do not share a lane with large ones)
        job.team = team if lane == "items" else 1
        self.team_sizes_used.add(job.team)
        job.group = f"{group}-t{job.team}-{(need - 4096).bit_length()}"
        if self.keep_series:
            job.series = {name: np.empty((req.sweeps, w) if w > 1 else req.sweeps, dtype=dt)
                          for name, dt, w in fields}
        else:
            job.series = {name: np.zeros(w, dtype=dt) for name, dt, w in fields}
            # error bars without keeping the series: streaming Gamma-method sums per scalar field
            if self.stats_lag > 0:
                job.stream = {name: HostStreamStats(self.stats_lag) for name, _, w in fields if w == 1}
        return job

    # ---- ticks -----------------------------------------------------------
    def _sweep_seconds(self, job: _Job) -> float:
        a, b = self.costs[(job.lane, job.family) if job.team == 1 else (f"team{job.team}", job.family)]
        return job.sweeps_per_meas * (a + b * job.req.n_sites)

    def _plan(self, lane: _Lane):
        plan = []
        for j in lane.jobs:
            left = j.req.sweeps - j.launched
            if left <= 0:
                continue
            per = self._sweep_seconds(j) * lane.scale
            n = min(left, max(1, int(self.tick_s / per)))
            if lane.kind == "grid":
                n = min(n, GRID_MAX_MEAS)
            plan.append([j, n])
        if not plan:
            return [], 0.0
        predicted = max(self._sweep_seconds(j) * lane.scale * n for j, n in plan)
        return plan, predicted

    def _launch(self, lane: _Lane) -> bool:
        plan, predicted = self._plan(lane)
        if not plan:
            return False
        size = sum(_round_up(j.meas_bytes * n) for j, n in plan)
        seg = self.arena.alloc(size)
        if seg is None:
            return False
        s = lane.stream
        if self.admit_event is not None:
            s.wait_event(self.admit_event)
        start, end, done = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
                            torch.cuda.Event())
        start.record(s)
        base = ptr(self.arena.dev) + seg
        entries = []
        off = seg
        items = []
        for j, n in plan:
            entries.append((j, n, off))
            ptrs = []
            o = base + (off - seg)
            for _, _, w in j.fields:
                ptrs.append(o)
                o += 8 * w * n
            if lane.kind == "items":
                it = CritmcItem.from_buffer_copy(j.item)
                it.sweep0 = j.chain.sweep
                it.n_meas = n
                it.e_out, it.vec_out, it.aux_out = ptrs[0], ptrs[1], ptrs[-1]
                if j.family.startswith("on"):
                    it.sc_out, it.ss_out = ptrs[2], ptrs[3]
                items.append(it)
            else:
                self._grid_call(lane, j, n, ptrs)
            off = _round_up(off + j.meas_bytes * n)
        if items:
            slot = lane.n_ticks % 2
            need = len(items) * ctypes.sizeof(CritmcItem)
            if lane.staging[slot] is None or lane.staging[slot].numel() < need:
                lane.staging[slot] = torch.empty(max(need, 1 << 16), dtype=torch.uint8, pin_memory=True)
            if lane.item_buffer is None or lane.item_buffer.numel() < _lib.lib().critmc_items_buffer_bytes(len(items)):
                # grow with headroom; the old buffer is only replaced between ticks of this stream
                lane.item_buffer = empty_bytes(_lib.lib().critmc_items_buffer_bytes(2 * len(items) + 64), self.device)
            arr = (CritmcItem * len(items))(*items)
            launch_items(arr, self.device, lane.item_buffer, staging=lane.staging[slot], stream=s.cuda_stream)
        end.record(s)
        with torch.cuda.stream(s):
            self.arena.host[seg:seg + size].copy_(self.arena.dev[seg:seg + size], non_blocking=True)
        done.record(s)
        for j, n, _ in entries:
            j.launched += n
            j.chain.sweep += n * j.sweeps_per_meas
        lane.n_ticks += 1
        self.ticks += 1
        lane.inflight.append(_Tick(lane, entries, seg, size, predicted, start, end, done, self.ticks))
        return True

    def _grid_call(self, lane: _Lane, j: _Job, n: int, ptrs: list) -> None:
        s = lane.stream
        scratch = self._grid_scratch(s)
        c = j.chain
        lx, ly, lz = c.dims
        if j.family == "msc":
            _lib.call_on(self.device, "critmc_ising_msc_run", ptr(c.words), len(c.shape), lx, ly, lz, 1,
                         c.key.ctypes.data, j.tables.ctypes.data, 1, c.sweep, j.sched.ctypes.data, len(j.sched), n,
                         ptr(j.tensors["running"]), ptrs[0], ptrs[1], ptrs[2], ptr(scratch), 0, c.k_inline,
                         s.cuda_stream)
        else:
            betas, steps = j.tables
            _lib.call_on(self.device, "critmc_on_run_grid", ptr(c.spins), len(c.shape), lx, ly, lz, c.n, 1,
                         c.key.ctypes.data, betas.ctypes.data, steps.ctypes.data, 1, c.sweep, j.sched.ctypes.data,
                         len(j.sched), n, ptrs[0], ptrs[1], ptrs[2], ptrs[3], ptrs[4], ptr(scratch),
                         c.blocks_per_chain, s.cuda_stream)

    def _grid_scratch(self, stream: torch.cuda.Stream) -> torch.Tensor:
        key = stream.cuda_stream
        if key not in self.grid_scratch:
            lib = _lib.lib()
            need = max(lib.critmc_ising_msc_scratch_bytes(1, GRID_MAX_MEAS),
                       lib.critmc_on_grid_scratch_bytes(1, GRID_MAX_MEAS, 3, 3))
            self.grid_scratch[key] = empty_bytes(need, self.device)
        return self.grid_scratch[key]

    def _harvest(self, tick: _Tick) -> None:
        tick.done.synchronize()
        lane = tick.lane
        lane.inflight.popleft()
        gpu = tick.start.elapsed_time(tick.end) * 1e-3
        self.gpu_seconds += gpu
        if tick.predicted > 0 and gpu > 0:
            # damped correction of this lane's cost model
            lane.scale *= min(4.0, max(0.25, gpu / tick.predicted)) ** 0.5
        host = self.arena.host_np
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
                    if name in j.stream:
                        j.stream[name].update(v)
            j.harvested += n
            self.updates_done += n * j.sweeps_per_meas * j.req.n_sites
            if j.harvested == j.req.sweeps:
                self._finish(j, now)
        self.arena.release(tick.offset, tick.size)
        if lane.kind == "grid" and not lane.jobs and not lane.inflight:
            self.grid_lanes.remove(lane)

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
                     req.n_sites * j.sweeps_per_meas * req.sweeps,
                     {name: hs.result() for name, hs in j.stream.items()} if j.stream else None)
        self.active.remove(j)
        j.home.jobs.remove(j)
        self.in_use -= j.dev_bytes
        j.chain = None
        j.tensors.clear()
        if self.on_result is not None:
            self.on_result(res)
        else:
            self.results.append(res)

    # ---- driving ---------------------------------------------------------
    def step(self) -> bool:
        """Admit, harvest finished ticks, keep two ticks in flight per lane.

        Returns False when there is nothing left to do.
        """
        progress = self._admit()
        for lane in list(self._lanes()):
            while lane.inflight and lane.inflight[0].done.query():
                self._harvest(lane.inflight[0])
                progress = True
        for lane in list(self._lanes()):
            while len(lane.inflight) < 2 and self._launch(lane):
                progress = True
        busy = any(lane.inflight for lane in self._lanes())
        if not progress and busy:
            time.sleep(2e-4)  # nothing to do until a tick ends
        return bool(self.queue or self.active or busy)

    def run(self, requests=None) -> list[Result]:
        """Submit ``requests`` (in arrival order) and serve until all are done."""
        for r in requests or ():
            self.submit(r)
        while self.step():
            if not self.active and self.queue:
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

