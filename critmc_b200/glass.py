r"""Edwards-Anderson +-J spin glasses with parallel tempering on the GPU.

API of critmc ``src/critmc/glass.py``: ``EdwardsAnderson`` (one disorder
realisation), ``geometric_temperatures``, ``ParallelTempering(model,
temperatures, seed=..., sweeps_per_step=...).run(n_bins) -> TemperingRun``.
``SpinGlassCampaign`` runs many samples of one lattice in one launch (one
thread block per sample, both replica sets resident in shared memory);
``MultiSizeCampaign`` runs the samples of several lattice sizes in one
persistent launch.

Only bimodal (+-1) couplings map onto the replica multi-spin-coded kernel;
Gaussian disorder is refused.  For the same seed, the couplings and the
initial spins equal critmc's (same Generator calls), the Philox keys of the
two replica sets are drawn from the same Generator afterwards.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .device import ptr, require_cuda, stream_handle, to_host
from .lattice import Lattice
from .rng import make_rng, philox_key

__all__ = ["EdwardsAnderson", "TemperingRun", "ParallelTempering", "SpinGlassCampaign", "MultiSizeCampaign",
           "geometric_temperatures", "OBS_E", "OBS_QL", "OBS_Q", "OBS_Q2", "OBS_Q4", "OBS_QK2",
           "OBS_COUNT", "N_OBS"]

# columns of acc[bin, temperature, :] (critmc kernels/glass.py:24-31)
OBS_E, OBS_QL, OBS_Q, OBS_Q2, OBS_Q4, OBS_QK2, OBS_COUNT = range(7)
N_OBS = 7
SWAP_WIDTH = 2048


class EdwardsAnderson:
    """One disorder realisation with +-1 couplings (critmc glass.py:45-90).

    The default disorder is critmc's, ``"gaussian"``, which the multi-spin-coded
    kernel cannot run: a sample without explicit couplings must ask for
    ``disorder="bimodal"``, so that ``EdwardsAnderson(lat, seed=s)`` never
    builds a different model from the one critmc builds for the same call.
    """

    def __init__(self, lattice: Lattice, couplings: np.ndarray | None = None, *,
                 disorder: str = "gaussian", seed=None):
        self.lattice = lattice
        self.disorder = disorder
        if not lattice.hypercubic or not lattice.bipartite or lattice.dim not in (2, 3):
            raise ValueError("the GPU spin-glass kernel needs a 2D/3D hypercubic lattice with even extents")
        if lattice.n_sites > 4096:
            raise ValueError("at most 4096 sites per sample")
        if len(set(lattice.shape)) != 1:
            raise ValueError("the GPU spin-glass kernel needs equal extents")
        if couplings is None:
            if disorder == "gaussian":
                raise ValueError("Gaussian couplings (critmc's default disorder) are not supported: the "
                                 "multi-spin-coded kernel runs +-J couplings only; pass disorder=\"bimodal\"")
            if disorder != "bimodal":
                raise ValueError(f"disorder is 'bimodal' (or 'gaussian' in critmc), not {disorder!r}")
            # +-1 with probability 1/2 each: one uniform index per bond into (-1, +1),
            # the draw critmc makes for a seed (glass.py:62-63)
            signs = np.array([-1.0, 1.0])
            couplings = signs[make_rng(seed).integers(0, 2, size=lattice.n_bonds)]
        table = np.array(couplings, dtype=np.float64)
        if table.shape != (lattice.n_bonds,):
            raise ValueError(f"one coupling per bond ({lattice.n_bonds}) is needed, got shape {table.shape}")
        if np.any(np.abs(table) != 1.0):
            raise ValueError("the multi-spin-coded kernel needs couplings of +-1")
        self.couplings = table

    @property
    def n_sites(self) -> int:
        return self.lattice.n_sites

    def energy(self, state: np.ndarray) -> float:
        """E = -sum over bonds of J_ij s_i s_j."""
        spins = np.asarray(state, dtype=np.float64)
        i, j = self.lattice.bonds.T
        return -float(np.sum(self.couplings * spins[i] * spins[j]))

    def coupling_bits(self) -> np.ndarray:
        """Per-slot bit masks of negative couplings in the device layout."""
        shape = self.lattice.shape
        dims = tuple(shape) + (1,) * (3 - len(shape))
        out = np.zeros(self.n_sites, dtype=np.uint8)
        _lib.call("critmc_ea_coupling_bits", len(shape), *dims,
                  np.ascontiguousarray(self.couplings).ctypes.data, out.ctypes.data)
        return out


def geometric_temperatures(t_min: float, t_max: float, n: int) -> np.ndarray:
    """``n`` temperatures from ``t_min`` to ``t_max`` with a constant ratio (critmc glass.py:93-95)."""
    ratio = t_max / t_min
    return t_min * np.power(ratio, np.arange(n) / (n - 1))


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
        """The last (longest, most equilibrated) bin of every observable."""
        return {name: series[-1] for name, series in self.bin_means().items()}


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
        temps = -np.sort(-np.asarray(temperatures, dtype=np.float64))  # hottest first
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
        n_steps = (1 << n_bins) - 1 if n_steps is None else int(n_steps)
        out = self._outputs(n_bins)
        shape = self.lattice.shape
        dims = tuple(shape) + (1,) * (3 - len(shape))
        t0 = time.perf_counter()
        _lib.call_on(self.device, "critmc_ea_pt_run", ptr(self.words), ptr(self.jneg), len(shape), *dims,
                     len(self.temperatures), self.n_samples, self.keys.ctypes.data, self.betas.ctypes.data,
                     ptr(self.swap_thr), SWAP_WIDTH, ptr(self.conf_at), ptr(self.labels), self.step, n_steps, n_bins,
                     self.sweeps_per_step, *(ptr(out[k]) for k in _OUT_KEYS), stream_handle(self.device))
        torch.cuda.synchronize(self.device)
        self.step += n_steps
        return self._collect(out, n_bins, time.perf_counter() - t0)

    def _outputs(self, n_bins: int) -> dict[str, torch.Tensor]:
        S, m, dev = self.n_samples, len(self.temperatures), self.device
        return {"acc": torch.zeros((S, n_bins, m, N_OBS), dtype=torch.float64, device=dev),
                "swap_acc": torch.zeros((S, m - 1), dtype=torch.int64, device=dev),
                "swap_try": torch.zeros((S, m - 1), dtype=torch.int64, device=dev),
                "label_hist": torch.zeros((S, m, 2), dtype=torch.int64, device=dev),
                "trips": torch.zeros((S, 2), dtype=torch.int64, device=dev)}

    def _collect(self, out: dict, n_bins: int, wall: float) -> list[TemperingRun]:
        acc_h, sa, st = to_host(out["acc"]), to_host(out["swap_acc"]), to_host(out["swap_try"])
        lh, tr = to_host(out["label_hist"]), to_host(out["trips"])
        with np.errstate(invalid="ignore", divide="ignore"):
            rate = sa / st
        return [TemperingRun(self.temperatures.copy(), self.lattice.n_sites, self.lattice.z, acc_h[i], rate[i],
                             lh[i], tr[i], wall / self.n_samples,
                             {"n_bins": n_bins, "sweeps_per_step": self.sweeps_per_step, "backend": "cuda"})
                for i in range(self.n_samples)]

    def spins(self) -> np.ndarray:
        """(samples, 2, m, N) spins per temperature index (critmc site order)."""
        w = to_host(self.words, np.uint32)
        return np.stack([_unpack_words(w[i], len(self.temperatures), self.lattice.shape)
                         for i in range(self.n_samples)])


_OUT_KEYS = ("acc", "swap_acc", "swap_try", "label_hist", "trips")


class _EaSize(ctypes.Structure):
    """Mirror of ``critmc_ea_size`` in include/critmc_b200.h."""

    _fields_ = [("words", ctypes.c_void_p), ("jneg", ctypes.c_void_p), ("keys", ctypes.c_void_p),
                ("conf_at", ctypes.c_void_p), ("labels", ctypes.c_void_p), ("acc", ctypes.c_void_p),
                ("swap_acc", ctypes.c_void_p), ("swap_try", ctypes.c_void_p), ("label_hist", ctypes.c_void_p),
                ("trips", ctypes.c_void_p), ("lx", ctypes.c_int32), ("ly", ctypes.c_int32),
                ("lz", ctypes.c_int32), ("n_samples", ctypes.c_int32)]


class MultiSizeCampaign:
    """Samples of several lattice sizes advanced by ONE persistent launch.

    ``campaigns``: one ``SpinGlassCampaign`` per size, all with the same
    temperatures, dimension and sweeps per step.  Thread blocks take (size,
    sample) items from a queue, largest lattices first, so the uneven sizes
    share the GPU without one launch per size; each sample's result equals
    its own campaign's ``run``.
    """

    def __init__(self, campaigns: list["SpinGlassCampaign"]):
        if not campaigns:
            raise ValueError("no campaigns")
        c0 = campaigns[0]
        for c in campaigns[1:]:
            if (not np.array_equal(c.temperatures, c0.temperatures) or c.lattice.dim != c0.lattice.dim
                    or c.sweeps_per_step != c0.sweeps_per_step or c.device != c0.device):
                raise ValueError("campaigns must share temperatures, dimension, sweeps per step and device")
            if c.step != c0.step:
                raise ValueError("campaigns must be at the same PT step")
        self.campaigns = campaigns
        self.device = c0.device
        self._dkeys = [torch.from_numpy(c.keys.reshape(-1).view(np.int32).copy()).to(self.device)
                       for c in campaigns]
        total = sum(c.n_samples for c in campaigns)
        self._bytes = _lib.lib().critmc_ea_campaign_buffer_bytes(len(campaigns), total)
        self._buffer = torch.empty(self._bytes, dtype=torch.uint8, device=self.device)
        self._staging = torch.empty(self._bytes, dtype=torch.uint8, pin_memory=True)

    @property
    def n_updates_per_step(self) -> int:
        """Attempted spin updates of one PT step (every temperature of both replica sets)."""
        return sum(c.n_samples * 2 * len(c.temperatures) * c.lattice.n_sites * c.sweeps_per_step
                   for c in self.campaigns)

    def launch(self, n_bins: int, n_steps: int | None = None, stream=None, control=None) -> list[dict]:
        """Enqueue ``n_steps`` PT steps of every sample (no synchronisation); returns the outputs.

        ``control``: an armed ``RunControl`` bounding the launch (None: runs to completion)."""
        n_steps = (1 << n_bins) - 1 if n_steps is None else int(n_steps)
        c0 = self.campaigns[0]
        outs = [c._outputs(n_bins) for c in self.campaigns]
        sizes = (_EaSize * len(self.campaigns))()
        for z, c, o, k in zip(sizes, self.campaigns, outs, self._dkeys):
            dims = tuple(c.lattice.shape) + (1,) * (3 - c.lattice.dim)
            z.words, z.jneg, z.keys = ptr(c.words), ptr(c.jneg), ptr(k)
            z.conf_at, z.labels = ptr(c.conf_at), ptr(c.labels)
            z.acc, z.swap_acc, z.swap_try = ptr(o["acc"]), ptr(o["swap_acc"]), ptr(o["swap_try"])
            z.label_hist, z.trips = ptr(o["label_hist"]), ptr(o["trips"])
            z.lx, z.ly, z.lz = dims
            z.n_samples = c.n_samples
        _lib.call_on(self.device, "critmc_ea_campaign_run_ctl", ctypes.cast(sizes, ctypes.c_void_p),
                     len(self.campaigns), c0.lattice.dim, len(c0.temperatures), c0.betas.ctypes.data,
                     ptr(c0.swap_thr), SWAP_WIDTH, c0.step, n_steps, n_bins, c0.sweeps_per_step, ptr(self._buffer),
                     self._bytes, self._staging.data_ptr(), control.handle if control is not None else None,
                     stream if stream is not None else stream_handle(self.device))
        for c in self.campaigns:
            c.step += n_steps
        return outs

    def run(self, n_bins: int, n_steps: int | None = None, control=None) -> list[list[TemperingRun]]:
        """Run every size; returns one list of ``TemperingRun`` per campaign.

        With an armed ``control`` the launch is bounded: ``RunStopped`` is raised
        when it ran out of its budget or was cancelled (outputs incomplete)."""
        t0 = time.perf_counter()
        outs = self.launch(n_bins, n_steps, control=control)
        torch.cuda.synchronize(self.device)
        if control is not None:
            control.wait(raise_on_stop=True)
        wall = time.perf_counter() - t0
        return [c._collect(o, n_bins, wall) for c, o in zip(self.campaigns, outs)]


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
