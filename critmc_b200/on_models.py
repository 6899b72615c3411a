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
        dev = self.device
        n, dim = self.n, len(self.shape)
        sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
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
            _lib.call("critmc_on_run_grid", *args, ptr(self._scratch), self.blocks_per_chain, stream_handle(dev))
        else:
            _lib.call("critmc_on_run", *args, stream_handle(dev))
        self.sweep += int(sched[:, 1].sum()) * n_meas
        return {"E": to_host(e)[0], "M": to_host(m)[0], "stiff_c": to_host(sc)[0],
                "stiff_s": to_host(ss)[0], "aux": to_host(aux)[0]}
