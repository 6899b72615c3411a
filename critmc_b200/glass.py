r"""Edwards-Anderson +-J spin glasses with parallel tempering on the GPU.

API of critmc ``src/critmc/glass.py``: ``EdwardsAnderson`` (one disorder
realisation), ``geometric_temperatures``, ``ParallelTempering(model,
temperatures, seed=..., sweeps_per_step=...).run(n_bins) -> TemperingRun``.
``SpinGlassCampaign`` runs many samples of one lattice in one launch (one
thread block per sample, both replica sets resident in shared memory).

Only bimodal (+-1) couplings map onto the replica multi-spin-coded kernel;
Gaussian disorder is refused.  For the same seed, the couplings and the
initial spins equal critmc's (same Generator calls), the Philox keys of the
two replica sets are drawn from the same Generator afterwards.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .device import ptr, require_cuda, stream_handle, to_host
from .lattice import Lattice
from .rng import make_rng, philox_key

__all__ = ["EdwardsAnderson", "TemperingRun", "ParallelTempering", "SpinGlassCampaign",
           "geometric_temperatures", "OBS_E", "OBS_QL", "OBS_Q", "OBS_Q2", "OBS_Q4", "OBS_QK2",
           "OBS_COUNT", "N_OBS"]

# columns of acc[bin, temperature, :] (critmc kernels/glass.py:24-31)
OBS_E, OBS_QL, OBS_Q, OBS_Q2, OBS_Q4, OBS_QK2, OBS_COUNT = range(7)
N_OBS = 7
SWAP_WIDTH = 2048


class EdwardsAnderson:
    """One disorder realisation with +-1 couplings (critmc glass.py:45-90)."""

    def __init__(self, lattice: Lattice, couplings: np.ndarray | None = None, *,
                 disorder: str = "bimodal", seed=None):
        self.lattice = lattice
        self.disorder = disorder
        if not lattice.hypercubic or not lattice.bipartite or lattice.dim not in (2, 3):
            raise ValueError("the GPU spin-glass kernel needs a 2D/3D hypercubic lattice with even extents")
        if lattice.n_sites > 4096:
            raise ValueError("at most 4096 sites per sample")
        if len(set(lattice.shape)) != 1:
            raise ValueError("the GPU spin-glass kernel needs equal extents")
        if couplings is None:
            rng = make_rng(seed)
            if disorder == "bimodal":
                couplings = rng.choice([-1.0, 1.0], size=lattice.n_bonds)
            elif disorder == "gaussian":
                raise ValueError("Gaussian couplings are not supported by the +-J multi-spin-coded kernel")
            else:
                raise ValueError("disorder must be 'gaussian' or 'bimodal'")
        couplings = np.asarray(couplings, dtype=np.float64)
        if couplings.shape != (lattice.n_bonds,):
            raise ValueError("need one coupling per bond")
        if not np.all(np.abs(couplings) == 1.0):
            raise ValueError("couplings must be +-1")
        self.couplings = couplings

    @property
    def n_sites(self) -> int:
        return self.lattice.n_sites

    def energy(self, state: np.ndarray) -> float:
        b = self.lattice.bonds
        s = np.asarray(state, dtype=np.float64)
        return float(-np.sum(self.couplings * s[b[:, 0]] * s[b[:, 1]]))

    def coupling_bits(self) -> np.ndarray:
        """Per-slot bit masks of negative couplings in the device layout."""
        shape = self.lattice.shape
        dims = tuple(shape) + (1,) * (3 - len(shape))
        out = np.zeros(self.n_sites, dtype=np.uint8)
        _lib.call("critmc_ea_coupling_bits", len(shape), *dims,
                  np.ascontiguousarray(self.couplings).ctypes.data, out.ctypes.data)
        return out


def geometric_temperatures(t_min: float, t_max: float, n: int) -> np.ndarray:
    """critmc glass.py:93-95."""
    return t_min * (t_max / t_min) ** (np.arange(n) / (n - 1))


@dataclass
class TemperingRun:
    """Accumulated measurements of one disorder sample (critmc glass.py:98-131)."""

    temperatures: np.ndarray
    n_sites: int
    z: int
    acc: np.ndarray
    swap_rate: np.ndarray
    label_hist: np.ndarray
    trips: np.ndarray
    wall_time: float = 0.0
    meta: dict = field(default_factory=dict)

    def bin_means(self) -> dict[str, np.ndarray]:
        cnt = self.acc[:, :, OBS_COUNT]
        with np.errstate(invalid="ignore", divide="ignore"):
            return {name: self.acc[:, :, col] / cnt for name, col in (
                ("e", OBS_E), ("ql", OBS_QL), ("absq", OBS_Q), ("q2", OBS_Q2), ("q4", OBS_Q4),
                ("qk2", OBS_QK2))}

    def equilibrium(self) -> dict[str, np.ndarray]:
        return {k: v[-1] for k, v in self.bin_means().items()}


def _pack_words(spins: np.ndarray, shape) -> np.ndarray:
    """(2, m, N) int8 spins of the configurations at temperatures 0..m-1 ->
    (2, 2 * slots) uint32 words, bit k = temperature k, colour-major slots."""
    from .layout import checkerboard_order

    order = checkerboard_order(shape).reshape(-1)  # slot position -> site
    bits = (spins[:, :, order] > 0).astype(np.uint64)  # (2, m, sites)
    w = np.zeros((2, order.size), dtype=np.uint64)
    for k in range(spins.shape[1]):
        w |= bits[:, k, :] << np.uint64(k)
    return w.astype(np.uint32)


def _unpack_words(words: np.ndarray, m: int, shape) -> np.ndarray:
    from .layout import checkerboard_order

    order = checkerboard_order(shape).reshape(-1)
    out = np.empty((2, m, order.size), dtype=np.int8)
    for k in range(m):
        bits = ((words >> np.uint32(k)) & 1).astype(np.int8)
        out[:, k, order] = 2 * bits - 1
    return out


class SpinGlassCampaign:
    """Parallel tempering of many disorder samples of one lattice in one launch."""

    def __init__(self, models: list[EdwardsAnderson], temperatures, *, seeds=None,
                 sweeps_per_step: int = 1, device=None):
        if not models:
            raise ValueError("no samples")
        lat = models[0].lattice
        if any(md.lattice.shape != lat.shape for md in models):
            raise ValueError("all samples must share the lattice")
        temps = np.sort(np.asarray(temperatures, dtype=np.float64))[::-1]  # hot -> cold
        if not 2 <= len(temps) <= 32:
            raise ValueError("between 2 and 32 temperatures")
        self.device = require_cuda(device)
        self.models = models
        self.lattice = lat
        self.temperatures = temps
        self.betas = np.ascontiguousarray(1.0 / temps)
        self.sweeps_per_step = int(sweeps_per_step)
        m, n, S = len(temps), lat.n_sites, len(models)
        seeds = [None] * S if seeds is None else list(seeds)
        spins = np.empty((S, 2, m, n), dtype=np.int8)
        keys = np.empty((S, 2, 2), dtype=np.uint32)
        for i, sd in enumerate(seeds):
            rng = make_rng(sd)
            spins[i] = (2 * rng.integers(0, 2, size=(2, m, n)) - 1).astype(np.int8)  # glass.py:148
            keys[i, 0] = philox_key(rng)
            keys[i, 1] = philox_key(rng)
        self.keys = np.ascontiguousarray(keys)
        self.initial_spins = spins
        words = np.stack([_pack_words(spins[i], lat.shape) for i in range(S)])
        self.words = torch.from_numpy(words.view(np.int32)).to(self.device)
        jneg = np.stack([md.coupling_bits() for md in models])
        self.jneg = torch.from_numpy(jneg).to(self.device)
        self.conf_at = torch.from_numpy(np.tile(np.arange(m, dtype=np.uint8), (S, 2, 1))).to(self.device)
        self.labels = torch.zeros((S, 2, m), dtype=torch.uint8, device=self.device)
        table = np.zeros((m - 1, SWAP_WIDTH), dtype=np.uint32)
        _lib.call("critmc_pt_swap_table", m, self.betas.ctypes.data, SWAP_WIDTH, table.ctypes.data)
        self.swap_thr = torch.from_numpy(table.view(np.int32)).to(self.device)
        self.step = 0

    @property
    def n_samples(self) -> int:
        return len(self.models)

    def run(self, n_bins: int, n_steps: int | None = None) -> list[TemperingRun]:
        """Run ``2^n_bins - 1`` PT steps (or ``n_steps``), log-binned as critmc."""
        S, m = self.n_samples, len(self.temperatures)
        n_steps = (1 << n_bins) - 1 if n_steps is None else int(n_steps)
        dev = self.device
        acc = torch.zeros((S, n_bins, m, N_OBS), dtype=torch.float64, device=dev)
        swap_acc = torch.zeros((S, m - 1), dtype=torch.int64, device=dev)
        swap_try = torch.zeros((S, m - 1), dtype=torch.int64, device=dev)
        label_hist = torch.zeros((S, m, 2), dtype=torch.int64, device=dev)
        trips = torch.zeros((S, 2), dtype=torch.int64, device=dev)
        shape = self.lattice.shape
        dims = tuple(shape) + (1,) * (3 - len(shape))
        t0 = time.perf_counter()
        _lib.call("critmc_ea_pt_run", ptr(self.words), ptr(self.jneg), len(shape), *dims, m, S,
                  self.keys.ctypes.data, self.betas.ctypes.data, ptr(self.swap_thr), SWAP_WIDTH,
                  ptr(self.conf_at), ptr(self.labels), self.step, n_steps, n_bins,
                  self.sweeps_per_step, ptr(acc), ptr(swap_acc), ptr(swap_try), ptr(label_hist),
                  ptr(trips), stream_handle(dev))
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
        self.step += n_steps
        acc_h, sa, st = to_host(acc), to_host(swap_acc), to_host(swap_try)
        lh, tr = to_host(label_hist), to_host(trips)
        runs = []
        with np.errstate(invalid="ignore", divide="ignore"):
            rate = sa / st
        for i in range(S):
            runs.append(TemperingRun(self.temperatures.copy(), self.lattice.n_sites, self.lattice.z,
                                     acc_h[i], rate[i], lh[i], tr[i], wall / S,
                                     {"n_bins": n_bins, "sweeps_per_step": self.sweeps_per_step,
                                      "backend": "cuda"}))
        return runs

    def spins(self) -> np.ndarray:
        """(samples, 2, m, N) spins per temperature index (critmc site order)."""
        w = to_host(self.words, np.uint32)
        return np.stack([_unpack_words(w[i], len(self.temperatures), self.lattice.shape)
                         for i in range(self.n_samples)])


class ParallelTempering:
    """Parallel tempering for one sample with two replica sets (critmc glass.py:134-208)."""

    def __init__(self, model: EdwardsAnderson, temperatures, *, seed=None,
                 sweeps_per_step: int = 1, device=None):
        self.model = model
        self._campaign = SpinGlassCampaign([model], temperatures, seeds=[seed],
                                           sweeps_per_step=sweeps_per_step, device=device)
        self.temperatures = self._campaign.temperatures
        self.betas = self._campaign.betas
        self.sweeps_per_step = self._campaign.sweeps_per_step

    def run(self, n_bins: int) -> TemperingRun:
        return self._campaign.run(n_bins)[0]
