"""Canonical Markov-chain driver with critmc's API (``src/critmc/sim.py``).

>>> from critmc_b200 import Simulation, Ising, square
>>> sim = Simulation(Ising(square(64)), beta=0.44, updates="metropolis", seed=1)
>>> sim.thermalize(2_000)
>>> ts = sim.run(20_000)
>>> ts["e"].mean(), ts["absm"].mean()

An update schedule is a ``+``-separated list of moves applied once per
measurement (``"metropolis"``, ``"heatbath+4*overrelax"``, ...), with critmc's
syntax (sim.py:112-131).  The chain's configuration stays on the GPU between
calls; ``Simulation.state`` copies it back on demand.  Every random number is a
function of (Philox key, sweep index, site), so a chain's streams do not depend
on how ``run`` splits the work into chunks (critmc tests/test_sim_chunks.py
checks the same property).
"""

from __future__ import annotations

import math
import re
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any

import numpy as np

from .io import load_npz, save_npz
from .models import (
    AUX_ACCEPTED,
    AUX_WOLFF_SIZE,
    HEATBATH,
    METROPOLIS,
    METROPOLIS_RANDOM,
    OVERRELAX,
    SWENDSEN_WANG,
    UPDATE_CODES,
    WOLFF,
    Model,
    derive,
)
from .rng import make_rng

__all__ = ["TimeSeries", "Simulation", "parse_updates"]

_SINGLE_SITE = (METROPOLIS, METROPOLIS_RANDOM)
_SWEEPS = (METROPOLIS, METROPOLIS_RANDOM, HEATBATH, OVERRELAX, SWENDSEN_WANG)  # one visit of every site each


@dataclass
class TimeSeries:
    """Measurement streams of one chain (``raw``) and their metadata (critmc sim.py:49-110).

    Indexing gives a raw stream or a per-site observable derived from the raw
    ones (``e``, ``m``, ``m2``, ``absm``, ...).
    """

    raw: dict[str, np.ndarray]
    meta: dict[str, Any]
    _derived: dict[str, np.ndarray] = field(default_factory=dict, repr=False)

    def _observables(self) -> dict[str, np.ndarray]:
        if not self._derived:
            self._derived = derive(self.raw, self.meta)
        return self._derived

    def __len__(self) -> int:
        return len(self.raw["E"])

    def __getitem__(self, key: str) -> np.ndarray:
        if key in self.raw:
            return self.raw[key]
        table = self._observables()
        if key not in table:
            raise KeyError(f"{key!r} is neither a raw stream nor a derived observable; known: {self.keys()}")
        return table[key]

    def keys(self) -> list[str]:
        return sorted({*self.raw, *self._observables()})

    @property
    def beta(self) -> float:
        return float(self.meta["beta"])

    @property
    def n_sites(self) -> int:
        return int(self.meta["N"])

    @property
    def L(self) -> int:
        return int(self.meta["L"])

    def slice(self, start: int | None = None, stop: int | None = None) -> TimeSeries:
        """Measurements ``start:stop`` with the same metadata."""
        window = slice(start, stop)
        return TimeSeries({name: stream[window] for name, stream in self.raw.items()}, dict(self.meta))

    @staticmethod
    def concatenate(parts: list[TimeSeries]) -> TimeSeries:
        """The parts one after the other; the metadata of the first, with the total count."""
        if len(parts) == 0:
            raise ValueError("concatenate needs at least one time series")
        names = list(parts[0].raw)
        joined = {name: np.concatenate([part.raw[name] for part in parts]) for name in names}
        meta = {**parts[0].meta, "n_meas": int(sum(map(len, parts)))}
        return TimeSeries(joined, meta)

    def save(self, path: str | Path) -> Path:
        return save_npz(path, self.raw, self.meta)

    @classmethod
    def load(cls, path: str | Path) -> TimeSeries:
        arrays, meta = load_npz(path)
        return cls(arrays, meta)


_TERM = re.compile(r"(?:(?P<count>[^*]*)\*)?(?P<name>.*)")


def parse_updates(updates: str) -> list[tuple[str, int | None]]:
    """``"heatbath+4*overrelax"`` -> ``[("heatbath", None), ("overrelax", 4)]`` (critmc sim.py:112-131).

    Whitespace and case are ignored and empty terms skipped; ``None`` means the
    move's default count (one sweep; for ``wolff``, tuned during thermalisation).
    """
    terms = [t for t in re.sub(r"\s+", "", updates).lower().split("+") if t]
    if not terms:
        raise ValueError(f"no moves in the update string {updates!r}")
    rows: list[tuple[str, int | None]] = []
    for term in terms:
        parts = _TERM.fullmatch(term)
        count, name = parts["count"], parts["name"]
        if count is not None and not (count.isdecimal() and int(count) > 0):
            raise ValueError(f"the count in {term!r} is not a positive integer")
        rows.append((name, int(count) if count is not None else None))
    unknown = sorted({name for name, _ in rows} - set(UPDATE_CODES))
    if unknown:
        raise ValueError(f"unknown moves {unknown}; the moves are {sorted(UPDATE_CODES)}")
    return rows


class Simulation:
    """A single Markov chain at fixed inverse temperature ``beta``, run on the GPU.

    The parameters are critmc's (sim.py:134-181): ``seed`` an int, SeedSequence or
    Generator; ``start`` "random" (hot) or "ordered" (cold); ``state`` an initial
    configuration to copy.  ``device`` selects the CUDA device.
    """

    def __init__(self, model: Model, beta: float, updates: str = "metropolis", *, seed: Any = None,
                 start: str = "random", state: np.ndarray | None = None, device=None):
        rows = parse_updates(updates)
        model.check_updates([row[0] for row in rows])
        self.model = model
        self.beta = float(beta)
        self.updates = updates
        self.seed = int(seed) if isinstance(seed, (int, np.integer)) else None  # as recorded in the metadata
        self.rng = make_rng(seed)
        self.schedule = np.array([(UPDATE_CODES[name], count or 1) for name, count in rows], dtype=np.int64)
        # rows "wolff" without a count: their count follows N / <|C|> during thermalisation
        self._tuned_wolff_rows = [r for r, (name, count) in enumerate(rows) if name == "wolff" and count is None]
        self._mean_cluster = math.nan
        self._wolff_history: list[int] = []
        if state is None:
            first = model.initial_state(start, self.rng)
            self.start = start
        else:
            first = np.array(state, copy=True)
            self.start = "given"
        self.running = model.begin(first)
        self.chain = model.to_device(first, self.rng, device)
        self.n_therm = 0
        self.n_meas = 0

    @property
    def state(self) -> np.ndarray:
        """The current configuration, copied from the device (critmc site order)."""
        return self.chain.fetch()

    def _count(self, *codes: int) -> int:
        """Moves per measurement of the given kinds in the current schedule."""
        return int(sum(reps for code, reps in self.schedule if code in codes))

    def _advance(self, n_meas: int) -> dict[str, np.ndarray]:
        return self.model.advance(self.chain, self.running, self.beta, self.schedule, n_meas)

    def _retune_wolff(self, aux: np.ndarray) -> None:
        """Mean cluster size from the later half of a chunk; tuned rows move towards
        N / <|C|>, by at most a factor 4 per chunk (a hot start has tiny clusters)."""
        per_meas = self._count(WOLFF)
        later = aux[len(aux) // 2:, AUX_WOLFF_SIZE]
        self._mean_cluster = float(later.sum() / (per_meas * len(later)))
        if not self._tuned_wolff_rows or self._mean_cluster <= 0:
            return
        goal = max(1, int(round(self.model.n_sites / self._mean_cluster)))
        for row in self._tuned_wolff_rows:
            now = int(self.schedule[row, 1])
            self.schedule[row, 1] = min(max(goal, max(1, now // 4)), 4 * now)
        self._wolff_history.append(int(self.schedule[self._tuned_wolff_rows[0], 1]))

    def _retune_step(self, aux: np.ndarray) -> None:
        """Scale the O(n) Metropolis step by (acceptance / 0.5), within [0.5, 2] per chunk
        and [1e-3, 10] overall."""
        tries = self._count(*_SINGLE_SITE) * self.model.n_sites * len(aux)
        factor = min(max(aux[:, AUX_ACCEPTED].sum() / tries / 0.5, 0.5), 2.0)
        self.running["step"] = float(min(max(self.running["step"] * factor, 1e-3), 10.0))

    def thermalize(self, n_meas: int, *, tune: bool = True, n_chunks: int = 10) -> dict[str, Any]:
        """Discard ``n_meas`` measurements in up to ``n_chunks`` chunks, tuning the Wolff
        count and the O(n) Metropolis step after each (critmc sim.py:193-231)."""
        if n_meas < 0:
            raise ValueError(f"thermalize needs n_meas >= 0, got {n_meas}")
        chunks = max(1, min(n_chunks, n_meas))
        edges = np.linspace(0, n_meas, chunks + 1).astype(int)  # critmc's chunk boundaries
        single_site = self._count(*_SINGLE_SITE)
        for size in np.diff(edges):
            if size == 0:
                continue
            aux = self._advance(int(size))["aux"]
            if not tune:
                continue
            if self._count(WOLFF):
                self._retune_wolff(aux)
            if single_site and "step" in self.running:
                self._retune_step(aux)
        self.n_therm += int(n_meas)
        return self.tuning()

    def tuning(self) -> dict[str, Any]:
        """The adaptive parameters: schedule, Wolff count and mean cluster, O(n) step."""
        report: dict[str, Any] = {"schedule": self.schedule.tolist()}
        wolff = self._count(WOLFF)
        if wolff:
            report.update(wolff_per_meas=wolff, mean_cluster=self._mean_cluster)
            if self._wolff_history:
                report["wolff_history"] = list(self._wolff_history)
        if "step" in self.running:
            report["step"] = self.running["step"]
        return report

    def _collect(self, n_meas: int, chunk: int) -> dict[str, np.ndarray]:
        """``n_meas`` measurements, advanced ``chunk`` at a time into one set of streams."""
        first = self._advance(min(chunk, n_meas))
        if len(first["aux"]) == n_meas:
            return first
        streams = {name: np.empty((n_meas,) + part.shape[1:], dtype=part.dtype) for name, part in first.items()}
        done = 0
        part = first
        while True:
            k = len(part["aux"])
            for name, values in part.items():
                streams[name][done:done + k] = values
            done += k
            if done == n_meas:
                return streams
            part = self._advance(min(chunk, n_meas - done))

    def run(self, n_meas: int, *, chunk: int = 1 << 16) -> TimeSeries:
        """Record ``n_meas`` measurements (critmc sim.py:244-297)."""
        if n_meas < 1:
            raise ValueError(f"run needs n_meas >= 1, got {n_meas}")
        t0 = time.perf_counter()
        raw = self._collect(n_meas, chunk)
        wall = time.perf_counter() - t0
        self.n_meas += n_meas
        aux = raw["aux"]
        n = self.model.n_sites
        wolff = self._count(WOLFF)
        single_site = self._count(*_SINGLE_SITE)
        mean_cluster = float(aux[:, AUX_WOLFF_SIZE].sum() / (wolff * n_meas)) if wolff else float("nan")
        # a Wolff update counts as the fraction <|C|> / N of a sweep
        sweeps = self._count(*_SWEEPS) + (wolff * mean_cluster / n if wolff else 0.0)
        acceptance = float(aux[:, AUX_ACCEPTED].sum() / (single_site * n * n_meas)) if single_site else None
        meta = dict(self.model.meta())
        meta.update(beta=self.beta, updates=self.updates, schedule=self.schedule.tolist(), seed=self.seed,
                    start=self.start, n_therm=self.n_therm, n_meas=n_meas, sweeps_per_meas=float(sweeps),
                    mean_cluster=mean_cluster, acceptance=acceptance, step=self.running.get("step"), wall_time=wall,
                    site_updates_per_s=sweeps * n * n_meas / wall if wall > 0 else None, backend="cuda")
        return TimeSeries(raw, meta)
