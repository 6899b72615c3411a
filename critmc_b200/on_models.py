"""O(n) chains (XY, Heisenberg) with FP32 unit spins.

Two lanes give identical results: ``"block"`` (``critmc_on_run``, one thread
block per chain, lattice in shared memory when it fits) and ``"grid"``
(``critmc_on_run_grid``, many blocks per chain, one launch per colour,
replayed as CUDA graphs: lower latency for a large lattice).  ``lane="auto"``
takes the grid lane from ``GRID_MIN_SITES`` sites on.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import empty_bytes, ptr, require_cuda, stream_handle, to_host
from .layout import cb_pack, cb_unpack

N_AUX = 4
GRID_MIN_SITES = 4096
OVERRELAX = 5
CLUSTER_CODES = (3, 4)  # Wolff, Swendsen-Wang


class ONChain:
    """One O(n) chain: FP32 components, colour-major structure of arrays on the device."""

    def __init__(self, model, state: np.ndarray, key: np.ndarray, device, lane: str = "auto"):
        self.device = require_cuda(device)
        if lane not in ("auto", "block", "grid"):
            raise ValueError(f"lane must be auto, block or grid, got {lane!r}")
        self.model = model
        self.n = model.n
        self.shape = tuple(model.lattice.shape)
        self.dims = self.shape + (1,) * (3 - len(self.shape))
        self.key = np.ascontiguousarray(key, dtype=np.uint32).reshape(1, 2)
        s = np.asarray(state, dtype=np.float32).reshape(-1, self.n)
        comps = np.stack([cb_pack(s[:, k], self.shape) for k in range(self.n)])  # (n, 2, rows, hx)
        self.spins = torch.from_numpy(np.ascontiguousarray(comps)).to(self.device)
        self.sweep = 0
        n_sites = int(np.prod(self.shape))
        self.lane = lane if lane != "auto" else ("grid" if n_sites >= GRID_MIN_SITES else "block")
        self.blocks_per_chain = 0
        self._scratch = None

    def fetch(self) -> np.ndarray:
        comps = to_host(self.spins)
        out = np.stack([cb_unpack(comps[k], self.shape) for k in range(self.n)], axis=1)
        return out.astype(np.float64)

    def advance(self, running, beta, schedule, n_meas):
        sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
        if np.isin(sched[:, 0], CLUSTER_CODES).any():
            return self._advance_with_clusters(running, beta, sched, n_meas)
        return self._advance_sweeps(running, beta, sched, n_meas)

    def _advance_with_clusters(self, running, beta, sched, n_meas):
        """Schedules with Wolff / Swendsen-Wang rows (critmc kernels/on.py:349-418).

        Per measurement the rows run in order: consecutive sweep rows as one
        ``critmc_on_run`` call (which ends with a renormalisation and a
        measurement), cluster rows as ``critmc_on_cluster_update`` calls (the
        counter advances by one per update, as for sweeps); the measurement
        of the last call is the measurement of the row set, a zero-repetition
        call providing it after a trailing cluster row.  aux as critmc: accepted
        moves, summed Wolff size, SW sum |C|^2 and cluster count.
        """
        dev = self.device
        lx, ly, lz = self.dims
        n_sites = int(np.prod(self.shape))
        if getattr(self, "_cl_scratch", None) is None:
            self._cl_scratch = empty_bytes(_lib.lib().critmc_cluster_scratch_bytes(1, n_sites), dev)
        stats = torch.zeros((1, 3), dtype=torch.int64, device=dev)
        segments: list[tuple[str, np.ndarray]] = []
        pending: list[list[int]] = []
        for code, reps in sched:
            if code in CLUSTER_CODES:
                if pending:
                    segments.append(("sweeps", np.array(pending, dtype=np.int64)))
                    pending = []
                segments.append(("cluster", np.array([code, reps], dtype=np.int64)))
            else:
                pending.append([int(code), int(reps)])
        segments.append(("sweeps", np.array(pending or [[OVERRELAX, 0]], dtype=np.int64)))
        out = {k: [] for k in ("E", "M", "stiff_c", "stiff_s", "aux")}
        for _ in range(n_meas):
            stats.zero_()
            accepted = 0
            part = None
            for kind, seg in segments:
                if kind == "cluster":
                    for _ in range(int(seg[1])):
                        _lib.call_on(dev, "critmc_on_cluster_update", ptr(self.spins), len(self.shape), lx, ly, lz,
                                     self.n, 1, self.key.ctypes.data, float(beta), int(seg[0]), self.sweep,
                                     ptr(stats), ptr(self._cl_scratch), stream_handle(dev))
                        self.sweep += 1
                else:
                    part = self._advance_sweeps(running, beta, seg, 1)
                    accepted += int(part["aux"][0][0])
            st = to_host(stats).ravel()
            aux = np.array([accepted, st[0], st[1], st[2]], dtype=np.int64)
            for k in ("E", "M", "stiff_c", "stiff_s"):
                out[k].append(part[k][0])
            out["aux"].append(aux)
        return {k: np.array(v) for k, v in out.items()}

    def _advance_sweeps(self, running, beta, sched, n_meas):
        dev = self.device
        n, dim = self.n, len(self.shape)
        betas = np.array([beta], dtype=np.float64)
        steps = np.array([running.get("step", 1.0)], dtype=np.float64)
        e = torch.empty((1, n_meas), dtype=torch.float64, device=dev)
        m = torch.empty((1, n_meas, n), dtype=torch.float64, device=dev)
        sc = torch.empty((1, n_meas, dim), dtype=torch.float64, device=dev)
        ss = torch.empty((1, n_meas, dim), dtype=torch.float64, device=dev)
        aux = torch.empty((1, n_meas, N_AUX), dtype=torch.int64, device=dev)
        lx, ly, lz = self.dims
        args = (ptr(self.spins), dim, lx, ly, lz, n, 1, self.key.ctypes.data, betas.ctypes.data,
                steps.ctypes.data, 1, self.sweep, sched.ctypes.data, len(sched), n_meas, ptr(e), ptr(m),
                ptr(sc), ptr(ss), ptr(aux))
        if self.lane == "grid":
            need = _lib.lib().critmc_on_grid_scratch_bytes(1, n_meas, n, dim)
            if self._scratch is None or self._scratch.numel() < need:
                self._scratch = empty_bytes(need, dev)
            _lib.call_on(dev, "critmc_on_run_grid", *args, ptr(self._scratch), self.blocks_per_chain,
                         stream_handle(dev))
        else:
            _lib.call_on(dev, "critmc_on_run", *args, stream_handle(dev))
        self.sweep += int(sched[:, 1].sum()) * n_meas
        return {"E": to_host(e)[0], "M": to_host(m)[0], "stiff_c": to_host(sc)[0],
                "stiff_s": to_host(ss)[0], "aux": to_host(aux)[0]}


class ONEnsemble:
    """Many O(n) chains of one lattice advanced by one ``critmc_on_run`` call.

    ``temperatures`` x ``chains_per_temperature`` chains (chains of one
    temperature form a group), uniform random unit-vector starts; chain ``c``
    of temperature index ``t`` draws its start and Philox key from
    ``make_rng(seed, "on", n, L, t, c)``, so its trajectory does not depend on
    what it is batched with.  Replaces critmc's process pool over independent
    chains (src/critmc/runner.py:154-223) for the sampling step.
    """

    def __init__(self, model, temperatures, chains_per_temperature: int, *, seed: int = 0, step: float = 1.0,
                 device=None):
        from .rng import make_rng, philox_key

        self.device = require_cuda(device)
        self.model = model
        self.n = model.n
        self.shape = tuple(model.lattice.shape)
        self.dims = self.shape + (1,) * (3 - len(self.shape))
        self.betas = np.ascontiguousarray(1.0 / np.asarray(temperatures, dtype=np.float64))
        if not 1 <= len(self.betas) <= 16:
            raise ValueError("between 1 and 16 temperatures per ensemble")
        self.chains_per_temperature = int(chains_per_temperature)
        self.n_chains = len(self.betas) * self.chains_per_temperature
        keys, comps = [], []
        L = self.shape[0]
        for t in range(len(self.betas)):
            for c in range(self.chains_per_temperature):
                rng = make_rng(seed, "on", self.n, L, t, c)
                s = model.initial_state("random", rng).astype(np.float32)
                keys.append(philox_key(rng))
                comps.append(np.stack([cb_pack(s[:, k], self.shape) for k in range(self.n)]))
        self.keys = np.ascontiguousarray(np.stack(keys), dtype=np.uint32)
        self.spins = torch.from_numpy(np.ascontiguousarray(np.stack(comps))).to(self.device)
        self.steps = np.full(len(self.betas), float(step))
        self.sweep = 0

    @property
    def n_sites(self) -> int:
        return int(np.prod(self.shape))

    def run(self, n_meas: int, schedule, stream=None) -> dict[str, torch.Tensor]:
        """Apply ``schedule`` ((code, reps) rows) ``n_meas`` times to every chain; device outputs."""
        dev, n, dim = self.device, self.n, len(self.shape)
        sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
        nc = self.n_chains
        out = {"E": torch.empty((nc, n_meas), dtype=torch.float64, device=dev),
               "M": torch.empty((nc, n_meas, n), dtype=torch.float64, device=dev),
               "stiff_c": torch.empty((nc, n_meas, dim), dtype=torch.float64, device=dev),
               "stiff_s": torch.empty((nc, n_meas, dim), dtype=torch.float64, device=dev),
               "aux": torch.empty((nc, n_meas, N_AUX), dtype=torch.int64, device=dev)}
        lx, ly, lz = self.dims
        _lib.call_on(dev, "critmc_on_run", ptr(self.spins), dim, lx, ly, lz, n, nc, self.keys.ctypes.data,
                     self.betas.ctypes.data, self.steps.ctypes.data, len(self.betas), self.sweep, sched.ctypes.data,
                     len(sched), n_meas, *(ptr(out[k]) for k in ("E", "M", "stiff_c", "stiff_s")), ptr(out["aux"]),
                     stream if stream is not None else stream_handle(dev))
        self.sweep += int(sched[:, 1].sum()) * n_meas
        return out

    def chain(self, i: int) -> np.ndarray:
        """Configuration of chain ``i`` in critmc's site order, shape (N, n)."""
        comps = to_host(self.spins[i])
        return np.stack([cb_unpack(comps[k], self.shape) for k in range(self.n)], axis=1).astype(np.float64)
