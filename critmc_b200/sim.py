"""Canonical Markov-chain driver with critmc's API (``src/critmc/sim.py``).

>>> from critmc_b200 import Simulation, Ising, square
>>> sim = Simulation(Ising(square(64)), beta=0.44, updates="metropolis", seed=1)
>>> sim.thermalize(2_000)
>>> ts = sim.run(20_000)
>>> ts["e"].mean(), ts["absm"].mean()

An update schedule is a ``+``-separated list of moves applied once per
measurement (``"metropolis"``, ``"heatbath+4*overrelax"``, ...), parsed as in
critmc sim.py:112-131.  The chain's configuration stays on the GPU between
calls; ``Simulation.state`` copies it back on demand.  Every random number is
a function of (Philox key, sweep index, site), so a chain's streams do not
depend on how ``run`` splits the work into chunks (critmc
tests/test_sim_chunks.py checks the same property).
"""

from __future__ import annotations

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


@dataclass
class TimeSeries:
    """Raw measurement streams of one chain plus metadata (critmc sim.py:49-110)."""

    raw: dict[str, np.ndarray]
    meta: dict[str, Any]
    _derived: dict[str, np.ndarray] = field(default_factory=dict, repr=False)

    def __len__(self) -> int:
        return int(len(self.raw["E"]))

    def __getitem__(self, key: str) -> np.ndarray:
        if key in self.raw:
            return self.raw[key]
        if not self._derived:
            self._derived = derive(self.raw, self.meta)
        try:
            return self._derived[key]
        except KeyError:
            raise KeyError(f"no observable {key!r}; have {sorted(self.keys())}") from None

    def keys(self) -> list[str]:
        if not self._derived:
            self._derived = derive(self.raw, self.meta)
        return sorted(set(self.raw) | set(self._derived))

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
        return TimeSeries({k: v[start:stop] for k, v in self.raw.items()}, dict(self.meta))

    @staticmethod
    def concatenate(parts: list[TimeSeries]) -> TimeSeries:
        if not parts:
            raise ValueError("nothing to concatenate")
        raw = {k: np.concatenate([p.raw[k] for p in parts]) for k in parts[0].raw}
        meta = dict(parts[0].meta)
        meta["n_meas"] = sum(len(p) for p in parts)
        return TimeSeries(raw, meta)

    def save(self, path: str | Path) -> Path:
        return save_npz(path, self.raw, self.meta)

    @classmethod
    def load(cls, path: str | Path) -> TimeSeries:
        raw, meta = load_npz(path)
        return cls(raw, meta)


def parse_updates(updates: str) -> list[tuple[str, int | None]]:
    """``"heatbath+4*overrelax"`` -> ``[(name, count or None), ...]`` (critmc sim.py:112-131)."""
    rows: list[tuple[str, int | None]] = []
    for token in updates.replace(" ", "").lower().split("+"):
        if not token:
            continue
        if "*" in token:
            count, name = token.split("*", 1)
            if not count.isdecimal() or int(count) < 1:
                raise ValueError(f"repetition count must be a positive integer in {token!r}")
            rows.append((name, int(count)))
        else:
            rows.append((token, None))
    if not rows:
        raise ValueError("empty update schedule")
    unknown = [name for name, _ in rows if name not in UPDATE_CODES]
    if unknown:
        raise ValueError(f"unknown updates {unknown}; choose from {sorted(UPDATE_CODES)}")
    return rows


class Simulation:
    """A single Markov chain at fixed inverse temperature ``beta``, run on the GPU.

    Parameters follow critmc sim.py:134-181; ``device`` selects the CUDA device.
    """

    def __init__(self, model: Model, beta: float, updates: str = "metropolis", *, seed: Any = None,
                 start: str = "random", state: np.ndarray | None = None, device=None):
        rows = parse_updates(updates)
        model.check_updates([name for name, _ in rows])
        self.model = model
        self.beta = float(beta)
        self.updates = updates
        self.seed = seed if isinstance(seed, (int, np.integer)) else None
        self.rng = make_rng(seed)
        self.schedule = np.array(
            [[UPDATE_CODES[name], 1 if k is None else k] for name, k in rows], dtype=np.int64
        )
        # "wolff" without a count: tuned to about N / <|C|> clusters per measurement (sim.py:166, :208-222)
        self._auto_wolff = [r for r, (name, k) in enumerate(rows) if name == "wolff" and k is None]
        self._mean_cluster = float("nan")
        self._wolff_history: list[int] = []
        host_state = model.initial_state(start, self.rng) if state is None else np.array(state, copy=True)
        self.start = "given" if state is not None else start
        self.running = model.begin(host_state)
        self.chain = model.to_device(host_state, self.rng, device)
        self.n_therm = 0
        self.n_meas = 0

    @property
    def state(self) -> np.ndarray:
        """The current configuration, copied from the device (critmc site order)."""
        return self.chain.fetch()

    def _count(self, *codes: int) -> int:
        mask = np.isin(self.schedule[:, 0], codes)
        return int(self.schedule[mask, 1].sum())

    def _advance(self, n_meas: int) -> dict[str, np.ndarray]:
        return self.model.advance(self.chain, self.running, self.beta, self.schedule, n_meas)

    def thermalize(self, n_meas: int, *, tune: bool = True, n_chunks: int = 10) -> dict[str, Any]:
        """Discard ``n_meas`` measurements; tune the Wolff count and the O(n) Metropolis step
        (critmc sim.py:193-231)."""
        if n_meas < 0:
            raise ValueError("n_meas must not be negative")
        n_chunks = max(1, min(n_chunks, n_meas)) if n_meas else 1
        sizes = np.diff(np.linspace(0, n_meas, n_chunks + 1).astype(int))
        n_metro = self._count(METROPOLIS, METROPOLIS_RANDOM)
        n_wolff = self._count(WOLFF)
        for chunk in sizes:
            if chunk == 0:
                continue
            raw = self._advance(int(chunk))
            if not tune:
                continue
            aux = raw["aux"]
            if n_wolff:
                late = aux[len(aux) // 2:, AUX_WOLFF_SIZE]  # the better-equilibrated half
                mean_c = late.sum() / (n_wolff * len(late))
                self._mean_cluster = float(mean_c)
                if self._auto_wolff and mean_c > 0:
                    target = max(1, int(round(self.model.n_sites / mean_c)))
                    for row in self._auto_wolff:
                        current = int(self.schedule[row, 1])
                        # at most a factor 4 per chunk: a hot start has tiny clusters
                        self.schedule[row, 1] = int(np.clip(target, max(1, current // 4), 4 * current))
                    self._wolff_history.append(int(self.schedule[self._auto_wolff[0], 1]))
                    n_wolff = self._count(WOLFF)
            if "step" in self.running and n_metro:
                rate = aux[:, AUX_ACCEPTED].sum() / (n_metro * self.model.n_sites * len(aux))
                factor = float(np.clip(rate / 0.5, 0.5, 2.0))
                self.running["step"] = float(np.clip(self.running["step"] * factor, 1e-3, 10.0))
        self.n_therm += int(n_meas)
        return self.tuning()

    def tuning(self) -> dict[str, Any]:
        info: dict[str, Any] = {"schedule": self.schedule.tolist()}
        if self._count(WOLFF):
            info["wolff_per_meas"] = self._count(WOLFF)
            info["mean_cluster"] = self._mean_cluster
            if self._wolff_history:
                info["wolff_history"] = list(self._wolff_history)
        if "step" in self.running:
            info["step"] = self.running["step"]
        return info

    def run(self, n_meas: int, *, chunk: int = 1 << 16) -> TimeSeries:
        """Record ``n_meas`` measurements in chunks (critmc sim.py:244-297)."""
        if n_meas < 1:
            raise ValueError("n_meas must be positive")
        t0 = time.perf_counter()
        raw: dict[str, np.ndarray] = {}
        done = 0
        while done < n_meas:
            k = min(chunk, n_meas - done)
            part = self._advance(k)
            if k == n_meas:
                raw = part
            else:
                if not raw:
                    raw = {key: np.empty((n_meas, *v.shape[1:]), dtype=v.dtype) for key, v in part.items()}
                for key, v in part.items():
                    raw[key][done:done + k] = v
            done += k
        wall = time.perf_counter() - t0
        self.n_meas += n_meas
        aux = raw["aux"]
        n = self.model.n_sites
        n_wolff = self._count(WOLFF)
        mean_cluster = float(aux[:, AUX_WOLFF_SIZE].sum() / (n_wolff * n_meas)) if n_wolff else float("nan")
        sweeps = self._count(METROPOLIS, METROPOLIS_RANDOM, HEATBATH, OVERRELAX, SWENDSEN_WANG) + (
            n_wolff * mean_cluster / n if n_wolff else 0.0)
        n_single = self._count(METROPOLIS, METROPOLIS_RANDOM)
        meta = {
            **self.model.meta(),
            "beta": self.beta,
            "updates": self.updates,
            "schedule": self.schedule.tolist(),
            "seed": self.seed,
            "start": self.start,
            "n_therm": self.n_therm,
            "n_meas": n_meas,
            "sweeps_per_meas": float(sweeps),
            "mean_cluster": mean_cluster,
            "acceptance": (
                float(aux[:, AUX_ACCEPTED].sum() / (n_single * n * n_meas)) if n_single else None
            ),
            "step": self.running.get("step"),
            "wall_time": wall,
            "site_updates_per_s": sweeps * n * n_meas / wall if wall > 0 else None,
            "backend": "cuda",
        }
        return TimeSeries(raw, meta)


