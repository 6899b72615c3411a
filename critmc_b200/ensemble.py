"""Batches of independent chains advanced together on the GPU.

``IsingEnsemble`` holds ``len(betas) * chains_per_beta`` multi-spin-coded Ising
chains of one lattice in HBM (chains sharing a beta form a group) and
advances all of them with one kernel launch per half-sweep, replayed as CUDA
graphs.  Chain ``c`` of beta index ``b`` draws its Philox key from
``make_rng(seed, "ising", L, b, c)`` (critmc's spawn-key convention,
src/critmc/rng.py:28-66), so a chain's trajectory is the same whatever it is
batched with.  This replaces critmc's process pool over independent chains
(src/critmc/runner.py:154-223) for the sampling step.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .device import empty_bytes, ptr, require_cuda, stream_handle, to_dev, to_host
from .lattice import Lattice, square
from .layout import msc_unpack
from .models import HEATBATH, METROPOLIS, UPDATE_CODES, Ising, _msc_ok
from .rng import make_rng, philox_key
from .sim import parse_updates


@dataclass
class EnsembleSeries:
    """Per-chain series of one ``run`` call (host or device arrays)."""

    Eb: object  # (n_chains, n_meas) int64
    M: object
    aux: object  # (n_chains, n_meas, 4)


class IsingEnsemble:
    """Many Ising chains of one MSC-compatible lattice (2D/3D, lx a power-of-two multiple of 64)."""

    def __init__(self, lattice: Lattice | int, betas, chains_per_beta: int, *, h: float = 0.0,
                 seed: int = 0, start: str = "random", device=None, mode: int = 0,
                 k_inline: int = 8, tune: bool = False, philox_rounds: int = 10):
        self.lattice = square(lattice) if isinstance(lattice, int) else lattice
        shape = tuple(self.lattice.shape)
        if not (_msc_ok(shape) and self.lattice.bipartite):
            raise ValueError(f"{self.lattice!r} is not a multi-spin-coded lattice")
        self.device = require_cuda(device)
        self.model = Ising(self.lattice, h)
        self.betas = [float(b) for b in betas]
        if not 1 <= len(self.betas) <= 16:
            raise ValueError("between 1 and 16 betas per ensemble")
        self.chains_per_beta = int(chains_per_beta)
        self.n_chains = len(self.betas) * self.chains_per_beta
        self.shape = shape
        self.dims = shape + (1,) * (3 - len(shape))
        self.mode, self.k_inline = mode, k_inline
        if philox_rounds not in (10, 7):
            raise ValueError("philox_rounds is 10 (the library's stream) or 7 (the optional reduced-round planes)")
        # a different random stream, not a tuning knob: the acceptance planes from Philox4x32-7
        self.philox_rounds = philox_rounds
        self._stream_bits = 0x1000 if philox_rounds == 7 else 0
        L = shape[0]
        keys = [philox_key(make_rng(seed, "ising", L, b, c))
                for b in range(len(self.betas)) for c in range(self.chains_per_beta)]
        self.keys = np.ascontiguousarray(np.stack(keys), dtype=np.uint32)
        lx, ly, lz = self.dims
        rows = ly * lz
        self.words = torch.empty((self.n_chains, 2, rows, lx // 64), dtype=torch.int32, device=self.device)
        code = {"random": 0, "ordered": 1, "up": 1, "down": -1}[start]
        dkeys = to_dev(self.keys, self.device)
        st = stream_handle(self.device)
        _lib.call_on(self.device, "critmc_ising_msc_init", ptr(self.words), len(shape), lx, ly, lz, self.n_chains,
                     ptr(dkeys), code, st)
        self.running = torch.empty((self.n_chains, 2), dtype=torch.int64, device=self.device)
        _lib.call_on(self.device, "critmc_ising_msc_measure", ptr(self.words), len(shape), lx, ly, lz, self.n_chains,
                     ptr(self.running), st)
        self.tables = np.ascontiguousarray(np.stack([self.model.tables(b)[0] for b in self.betas]))
        self.sweep = 0
        self._scratch = None
        self._dev_out = None
        self.tuning = None
        if tune:
            # launch shape from the autotuner (cached per GPU, shape, batch): results do not change
            from .autotune import msc_mode, tune_msc

            self.tuning = tune_msc(shape, self.n_chains, beta=self.betas[0], h=h, device=self.device)
            self.mode = msc_mode(self.tuning["run"], self.tuning["mode"])
            self.k_inline = self.tuning["k_inline"]

    @property
    def n_sites(self) -> int:
        return self.lattice.n_sites

    def _schedule(self, updates: str) -> np.ndarray:
        rows = parse_updates(updates)
        self.model.check_updates([n for n, _ in rows])
        return np.array([[UPDATE_CODES[n], 1 if k is None else k] for n, k in rows], dtype=np.int64)

    def run(self, n_meas: int, updates: str = "metropolis", *, host: bool = True,
            out: EnsembleSeries | None = None) -> EnsembleSeries:
        """Apply ``updates`` ``n_meas`` times to every chain; returns the series.

        ``host=False`` keeps the series on the device; ``out`` reuses buffers
        (pinned host tensors when ``host``).
        """
        sched = self._schedule(updates)
        dev = self.device
        n = self.n_chains
        if host:
            # device outputs are staging only: reuse them from call to call
            if self._dev_out is None or self._dev_out[0].shape[1] != n_meas:
                self._dev_out = (torch.empty((n, n_meas), dtype=torch.int64, device=dev),
                                 torch.empty((n, n_meas), dtype=torch.int64, device=dev),
                                 torch.empty((n, n_meas, 4), dtype=torch.int64, device=dev))
            e, m, aux = self._dev_out
        else:  # returned to the caller: fresh tensors
            e = torch.empty((n, n_meas), dtype=torch.int64, device=dev)
            m = torch.empty((n, n_meas), dtype=torch.int64, device=dev)
            aux = torch.empty((n, n_meas, 4), dtype=torch.int64, device=dev)
        need = _lib.lib().critmc_ising_msc_scratch_bytes(n, n_meas)
        if self._scratch is None or self._scratch.numel() < need:
            self._scratch = empty_bytes(need, dev)
        lx, ly, lz = self.dims
        _lib.call_on(dev, "critmc_ising_msc_run", ptr(self.words), len(self.shape), lx, ly, lz, n,
                     self.keys.ctypes.data, self.tables.ctypes.data, len(self.betas), self.sweep, sched.ctypes.data,
                     len(sched), n_meas, ptr(self.running), ptr(e), ptr(m), ptr(aux), ptr(self._scratch),
                     self.mode | self._stream_bits, self.k_inline, stream_handle(dev))
        self.sweep += int(sched[:, 1].sum()) * n_meas
        if not host:
            return EnsembleSeries(e, m, aux)
        if out is None:
            out = EnsembleSeries(*(torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in (e, m, aux)))
        out.Eb.copy_(e, non_blocking=True)
        out.M.copy_(m, non_blocking=True)
        out.aux.copy_(aux, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return out

    def state(self, chain: int) -> np.ndarray:
        """Configuration of one chain in critmc's site order."""
        return msc_unpack(to_host(self.words[chain], np.uint32), self.shape)


_ = (METROPOLIS, HEATBATH)
