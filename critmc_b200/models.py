"""Spin models whose chains advance on the GPU.

Mirrors critmc ``src/critmc/models.py``: a model is a stateless description
(Hamiltonian on a lattice) that knows how to create states, which update
moves it supports, how to advance a chain, and how to derive per-site
observables (``derive``, critmc models.py:325-351).  The difference is where
the chain lives: ``to_device`` moves a configuration into the device layout
and ``advance`` runs the schedule there through the C ABI, returning the same
raw streams, keys and dtypes as critmc's numba ``run`` kernels.

Conventions (J = k_B = 1): Ising ``H = -sum s_i s_j - h sum s_i``,
Potts ``H = -sum delta(s_i, s_j)``, O(n) ``H = -sum S_i . S_j``.
"""

from __future__ import annotations

import ctypes
import math
from abc import ABC, abstractmethod
from typing import Any

import numpy as np
import torch

from . import _lib
from .device import empty_bytes, ptr, require_cuda, stream_handle, to_dev, to_host
from .layout import msc_pack, msc_unpack
from .lattice import Lattice, make_lattice
from .rng import philox_key

__all__ = ["Model", "Ising", "Potts", "ON", "XY", "Heisenberg", "build_model", "derive",
           "UPDATE_CODES", "N_AUX"]

# critmc kernels/common.py:16-31
METROPOLIS, METROPOLIS_RANDOM, HEATBATH, WOLFF, SWENDSEN_WANG, OVERRELAX = 0, 1, 2, 3, 4, 5
UPDATE_CODES = {
    "metropolis": METROPOLIS,
    "metropolis-random": METROPOLIS_RANDOM,
    "heatbath": HEATBATH,
    "wolff": WOLFF,
    "sw": SWENDSEN_WANG,
    "swendsen-wang": SWENDSEN_WANG,
    "overrelax": OVERRELAX,
}
AUX_ACCEPTED, AUX_WOLFF_SIZE, AUX_SW_C2, AUX_SW_NCLUSTERS = 0, 1, 2, 3
N_AUX = 4

# moves of critmc that are not data-parallel sweeps and stay on its CPU path
_NOT_ON_GPU = {
    "metropolis-random": "random-site Metropolis is a sequential walk, not a checkerboard sweep",
}
CLUSTER_CODES = (WOLFF, SWENDSEN_WANG)


def advance_with_clusters(model, chain, running, beta, schedule, n_meas, bits: bool, q: int):
    """``Model.advance`` for schedules with Wolff / Swendsen-Wang rows (Ising, Potts).

    Rows run in order once per measurement: sweep rows through the chain's own
    entry point, cluster rows through ``critmc_cluster_update`` on the chain's
    device lattice; the sweep counter advances by one per repetition of every
    row, as for sweeps.  aux columns as critmc (kernels/common.py:35-39).
    """
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    dev = chain.device
    potts = q > 0
    dims = chain.dims
    if not hasattr(chain, "_cl_scratch"):
        chain._cl_scratch = empty_bytes(_lib.lib().critmc_cluster_scratch_bytes(1, model.n_sites), dev)
    spins = chain.words if bits else chain.spins
    out_e = np.empty(n_meas, dtype=np.int64)
    out_m = np.empty((n_meas, q) if potts else n_meas, dtype=np.int64)
    aux = np.zeros((n_meas, N_AUX), np.int64)
    stats = torch.zeros((1, 3), dtype=torch.int64, device=dev)
    for meas in range(n_meas):
        stats.zero_()
        for code, reps in sched:
            if code in CLUSTER_CODES:
                if potts:
                    run_t = torch.tensor([running["energy"]], dtype=torch.int64, device=dev)
                    cnt_t = torch.from_numpy(np.asarray(running["counts"], dtype=np.int64)).to(dev)
                else:
                    run_t = torch.tensor([[running["e_b"], running["m"]]], dtype=torch.int64, device=dev)
                    cnt_t = None
                for _ in range(int(reps)):
                    _lib.call_on(dev, "critmc_cluster_update", int(bits), ptr(spins), len(chain.shape), *dims, q, 1,
                                 chain.key.ctypes.data, float(beta), int(code), chain.sweep, ptr(run_t), ptr(cnt_t),
                                 ptr(stats), ptr(chain._cl_scratch), stream_handle(dev))
                    chain.sweep += 1
                r = to_host(run_t).ravel()
                if potts:
                    running["energy"] = int(r[0])
                    running["counts"] = to_host(cnt_t).copy()
                else:
                    running["e_b"], running["m"] = int(r[0]), int(r[1])
            else:
                part = model._advance_sweeps(chain, running, beta, np.array([[code, reps]]), 1)
                aux[meas, AUX_ACCEPTED] += int(part["aux"][0][AUX_ACCEPTED])
        st = to_host(stats).ravel()
        aux[meas, AUX_WOLFF_SIZE] = st[0]
        aux[meas, AUX_SW_C2], aux[meas, AUX_SW_NCLUSTERS] = st[1], st[2]
        if potts:
            out_e[meas] = running["energy"]
            out_m[meas] = running["counts"]
        else:
            out_e[meas], out_m[meas] = running["e_b"], running["m"]
    if potts:
        return {"E": out_e, "counts": out_m, "aux": aux}
    h = model.h
    return {"E": out_e - h * out_m if h != 0.0 else out_e, "Eb": out_e, "M": out_m, "aux": aux}


def _checkerboard_shape(lattice: Lattice) -> tuple[int, ...]:
    if not lattice.hypercubic:
        raise ValueError(
            f"{lattice!r}: the GPU sweeps are checkerboard sweeps and need a bipartite "
            "hypercubic lattice (chain, square, cubic)"
        )
    if not lattice.bipartite:
        raise ValueError(f"{lattice!r}: checkerboard sweeps need every extent to be even")
    if lattice.dim > 3:
        raise ValueError("lattices of dimension > 3 are not supported on the GPU")
    return lattice.shape


class Model(ABC):
    """Base class of the GPU spin models (critmc models.py:32-92)."""

    kind: str = ""
    updates: tuple[str, ...] = ()

    def __init__(self, lattice: Lattice):
        self.lattice = lattice

    @property
    def n_sites(self) -> int:
        return self.lattice.n_sites

    @abstractmethod
    def initial_state(self, start: str, rng: np.random.Generator) -> np.ndarray: ...

    @abstractmethod
    def energy(self, state: np.ndarray) -> float: ...

    @abstractmethod
    def begin(self, state: np.ndarray) -> dict[str, Any]: ...

    @abstractmethod
    def to_device(self, state: np.ndarray, rng: np.random.Generator, device=None): ...

    @abstractmethod
    def advance(self, chain, running: dict[str, Any], beta: float, schedule: np.ndarray,
                n_meas: int) -> dict[str, np.ndarray]: ...

    def check_updates(self, names: list[str]) -> None:
        """Raise ValueError for moves this model does not run (with the reason where one is known)."""
        missing = [name for name in names if name not in set(self.updates)]
        if missing:
            reasons = [f"{name}: {_NOT_ON_GPU[name]}" for name in missing if name in _NOT_ON_GPU]
            detail = f" ({'; '.join(reasons)})" if reasons else ""
            raise ValueError(f"{type(self).__name__} on the GPU runs {list(self.updates)}, not {missing}{detail}")
        if self._binary and self.lattice.dim == 1 and "metropolis" in names:
            # On a ring a zero-energy flip is accepted with certainty; updating a whole
            # sublattice at once then moves every domain wall one site per half-sweep in
            # lockstep, walls never meet, and the chain is not ergodic.
            raise ValueError(
                "checkerboard metropolis is not ergodic for two-state spins on a ring; "
                "use heatbath"
            )

    @property
    def _binary(self) -> bool:
        return False

    def spec(self) -> dict[str, Any]:
        """What ``build_model`` needs to make this model again (critmc's model spec)."""
        return dict(model=self.kind, lattice=self.lattice.name, L=self.lattice.L)

    def meta(self) -> dict[str, Any]:
        """The spec plus the lattice's size, dimension and bond count (series metadata)."""
        lat = self.lattice
        return {**self.spec(), **dict(N=lat.n_sites, dim=lat.dim, n_bonds=lat.n_bonds)}

    def __repr__(self) -> str:
        return "{}({!r})".format(type(self).__name__, self.lattice)


def _msc_ok(shape: tuple[int, ...]) -> bool:
    lx = shape[0]
    wc = lx // 64
    return len(shape) in (2, 3) and lx % 64 == 0 and wc & (wc - 1) == 0


class _IsingMscChain:
    """One Ising chain in the multi-spin-coded layout."""

    def __init__(self, model: "Ising", state: np.ndarray, key: np.ndarray, device):
        self.device = require_cuda(device)
        self.shape = model.lattice.shape
        self.dims = tuple(self.shape) + (1,) * (3 - len(self.shape))
        self.words = to_dev(msc_pack(state, self.shape), self.device)
        self.key = np.ascontiguousarray(key, dtype=np.uint32).reshape(1, 2)
        self.sweep = 0
        self.mode = 0
        self.k_inline = 8

    @classmethod
    def on_device(cls, model: "Ising", key: np.ndarray, device, start: int = 0) -> "_IsingMscChain":
        """A chain whose configuration is drawn on the device (``critmc_ising_msc_init``)."""
        self = cls.__new__(cls)
        self.device = require_cuda(device)
        self.shape = model.lattice.shape
        self.dims = tuple(self.shape) + (1,) * (3 - len(self.shape))
        lx, ly, lz = self.dims
        self.words = torch.empty((2, ly * lz, lx // 64), dtype=torch.int32, device=self.device)
        self.key = np.ascontiguousarray(key, dtype=np.uint32).reshape(1, 2)
        self.sweep = 0
        self.mode = 0
        self.k_inline = 8
        dkey = to_dev(self.key, self.device)
        _lib.call_on(self.device, "critmc_ising_msc_init", ptr(self.words), len(self.shape), lx, ly, lz, 1, ptr(dkey),
                     start, stream_handle(self.device))
        return self

    def measure(self) -> torch.Tensor:
        """Device int64 (E_b, M) of the current configuration."""
        out = torch.empty((1, 2), dtype=torch.int64, device=self.device)
        lx, ly, lz = self.dims
        _lib.call_on(self.device, "critmc_ising_msc_measure", ptr(self.words), len(self.shape), lx, ly, lz, 1,
                     ptr(out), stream_handle(self.device))
        return out

    def fetch(self) -> np.ndarray:
        return msc_unpack(to_host(self.words, np.uint32), self.shape)


class Ising(Model):
    """Ising model with uniform field ``h`` (critmc models.py:95-162)."""

    kind = "ising"
    updates = ("metropolis", "heatbath", "wolff", "sw", "swendsen-wang")

    def __init__(self, lattice: Lattice, h: float = 0.0):
        super().__init__(lattice)
        if not math.isfinite(float(h)):
            raise ValueError(f"the field must be a finite number, got h = {h}")
        self.h = float(h)

    @property
    def _binary(self) -> bool:
        return True

    def initial_state(self, start, rng):
        """+-1 spins: "random" (a fair bit per site from ``rng``), "ordered"/"up", "down"."""
        fill = {"ordered": 1, "up": 1, "down": -1}
        if start == "random":
            bits = rng.integers(0, 2, size=self.n_sites)  # the draw of critmc's Ising start
            return np.where(bits == 1, 1, -1).astype(np.int8)
        if start not in fill:
            raise ValueError(f"start is 'random', 'ordered', 'up' or 'down', not {start!r}")
        return np.full(self.n_sites, fill[start], dtype=np.int8)

    def bond_energy(self, state) -> int:
        """E_b = -sum over bonds of s_i s_j."""
        spins = np.asarray(state, dtype=np.int64)
        i, j = self.lattice.bonds.T
        return -int(np.dot(spins[i], spins[j]))

    def energy(self, state):
        magnetisation = int(np.asarray(state, dtype=np.int64).sum())
        return float(self.bond_energy(state)) - self.h * magnetisation

    def begin(self, state):
        return {"e_b": self.bond_energy(state), "m": int(np.asarray(state, dtype=np.int64).sum())}

    def tables(self, beta: float) -> tuple[np.ndarray, int]:
        """``(2, 2, 16)`` uint32 class tables (metropolis, heat bath) and the spin flag."""
        z = self.lattice.z
        out = np.zeros((2, 2, 16), dtype=np.uint32)
        dep = 0
        for slot, algo in enumerate((METROPOLIS, HEATBATH)):
            flag = ctypes.c_int32(0)
            _lib.call("critmc_ising_class_table", algo, z, float(beta), self.h,
                      out[slot, 0].ctypes.data, out[slot, 1].ctypes.data, ctypes.byref(flag))
            if algo == METROPOLIS:
                dep = flag.value
        return out, dep

    def to_device(self, state, rng, device=None):
        shape = _checkerboard_shape(self.lattice)
        key = philox_key(rng)
        if _msc_ok(shape):
            return _IsingMscChain(self, np.asarray(state, dtype=np.int8), key, device)
        from .byte_models import IsingByteChain

        return IsingByteChain(self, np.asarray(state, dtype=np.int8), key, device)

    def advance(self, chain, running, beta, schedule, n_meas):
        if np.isin(np.asarray(schedule).reshape(-1, 2)[:, 0], CLUSTER_CODES).any():
            return advance_with_clusters(self, chain, running, beta, schedule, n_meas,
                                         isinstance(chain, _IsingMscChain), 0)
        return self._advance_sweeps(chain, running, beta, schedule, n_meas)

    def _advance_sweeps(self, chain, running, beta, schedule, n_meas):
        if not isinstance(chain, _IsingMscChain):
            return chain.advance(running, beta, schedule, n_meas)
        dev = chain.device
        tables, _ = self.tables(beta)
        sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
        run = torch.tensor([[running["e_b"], running["m"]]], dtype=torch.int64, device=dev)
        e = torch.empty((1, n_meas), dtype=torch.int64, device=dev)
        m = torch.empty((1, n_meas), dtype=torch.int64, device=dev)
        aux = torch.empty((1, n_meas, N_AUX), dtype=torch.int64, device=dev)
        scratch = empty_bytes(_lib.lib().critmc_ising_msc_scratch_bytes(1, n_meas), dev)
        lx, ly, lz = chain.dims
        _lib.call_on(dev, "critmc_ising_msc_run", ptr(chain.words), len(chain.shape), lx, ly, lz, 1,
                     chain.key.ctypes.data, tables.ctypes.data, 1, chain.sweep, sched.ctypes.data, len(sched), n_meas,
                     ptr(run), ptr(e), ptr(m), ptr(aux), ptr(scratch), chain.mode, chain.k_inline, stream_handle(dev))
        chain.sweep += int(sched[:, 1].sum()) * n_meas
        r = to_host(run)[0]
        running["e_b"], running["m"] = int(r[0]), int(r[1])
        e_b = to_host(e)[0]
        mm = to_host(m)[0]
        energy = e_b - self.h * mm if self.h != 0.0 else e_b
        return {"E": energy, "Eb": e_b, "M": mm, "aux": to_host(aux)[0]}

    def spec(self):
        return dict(super().spec(), h=self.h)


class Potts(Model):
    """q-state Potts model (critmc models.py:165-222)."""

    kind = "potts"
    updates = ("metropolis", "heatbath", "wolff", "sw", "swendsen-wang")

    def __init__(self, lattice: Lattice, q: int):
        super().__init__(lattice)
        if not 2 <= q <= 127:
            raise ValueError(f"Potts models here have 2 <= q <= 127 states, got q = {q}")
        self.q = int(q)

    @property
    def _binary(self) -> bool:
        return self.q == 2

    def initial_state(self, start, rng):
        """States 0..q-1: "random" (uniform per site from ``rng``) or "ordered"/"up" (all 0)."""
        if start == "random":
            return np.asarray(rng.integers(0, self.q, size=self.n_sites), dtype=np.int8)
        if start not in ("ordered", "up"):
            raise ValueError(f"start is 'random', 'ordered' or 'up', not {start!r}")
        return np.zeros(self.n_sites, dtype=np.int8)

    def bond_energy(self, state) -> int:
        """E = -(number of bonds whose ends agree)."""
        values = np.asarray(state)
        i, j = self.lattice.bonds.T
        return -int(np.count_nonzero(values[i] == values[j]))

    def energy(self, state):
        return float(self.bond_energy(state))

    def begin(self, state):
        counts = np.bincount(np.asarray(state, dtype=np.int64), minlength=self.q).astype(np.int64)
        return {"energy": self.bond_energy(state), "counts": counts}

    def to_device(self, state, rng, device=None):
        _checkerboard_shape(self.lattice)
        from .byte_models import PottsChain

        return PottsChain(self, np.asarray(state, dtype=np.int8), philox_key(rng), device)

    def advance(self, chain, running, beta, schedule, n_meas):
        if np.isin(np.asarray(schedule).reshape(-1, 2)[:, 0], CLUSTER_CODES).any():
            return advance_with_clusters(self, chain, running, beta, schedule, n_meas, False, self.q)
        return chain.advance(running, beta, schedule, n_meas)

    def _advance_sweeps(self, chain, running, beta, schedule, n_meas):
        return chain.advance(running, beta, schedule, n_meas)

    def spec(self):
        return dict(super().spec(), q=self.q)


class ON(Model):
    """Classical O(n) vector model with unit spins (critmc models.py:225-299)."""

    kind = "on"
    updates = ("metropolis", "heatbath", "overrelax", "wolff", "sw", "swendsen-wang")

    def __init__(self, lattice: Lattice, n: int):
        super().__init__(lattice)
        if n < 2:
            raise ValueError(f"O(n) models need n >= 2 components (n = 1 is Ising), got n = {n}")
        if n > 3:
            raise ValueError(f"the GPU O(n) kernels run n = 2 (XY) and n = 3 (Heisenberg), not n = {n}")
        self.n = int(n)

    def initial_state(self, start, rng):
        """Unit vectors: "random" (normalised Gaussian vectors from ``rng``, uniform on the
        sphere) or "ordered"/"up" (all along the first axis)."""
        if start == "random":
            v = rng.standard_normal((self.n_sites, self.n))
            return v / np.linalg.norm(v, axis=1)[:, None]
        if start not in ("ordered", "up"):
            raise ValueError(f"start is 'random', 'ordered' or 'up', not {start!r}")
        return np.eye(1, self.n).repeat(self.n_sites, axis=0)

    def energy(self, state):
        """E = -sum over bonds of S_i . S_j."""
        spins = np.asarray(state, dtype=np.float64)
        i, j = self.lattice.bonds.T
        return -float(np.einsum("bk,bk->", spins[i], spins[j]))

    def begin(self, state):
        return {"step": 1.0}

    def to_device(self, state, rng, device=None):
        _checkerboard_shape(self.lattice)
        from .on_models import ONChain

        return ONChain(self, np.asarray(state, dtype=np.float64), philox_key(rng), device)

    def advance(self, chain, running, beta, schedule, n_meas):
        return chain.advance(running, beta, schedule, n_meas)

    def spec(self):
        return dict(super().spec(), n=self.n)


def XY(lattice: Lattice) -> ON:
    return ON(lattice, 2)


def Heisenberg(lattice: Lattice) -> ON:
    return ON(lattice, 3)


def build_model(spec: dict[str, Any]) -> Model:
    """The model a spec names (``{"model": "ising", "lattice": "square", "L": 32, ...}``)."""
    lattice = make_lattice(spec["lattice"], int(spec["L"]))
    makers = {"ising": lambda: Ising(lattice, h=float(spec.get("h", 0.0))),
              "potts": lambda: Potts(lattice, int(spec["q"])),
              "on": lambda: ON(lattice, int(spec["n"]))}
    if spec["model"] not in makers:
        raise ValueError(f"model kind {spec['model']!r} is not one of {sorted(makers)}")
    return makers[spec["model"]]()


def derive(raw: dict[str, np.ndarray], meta: dict[str, Any]) -> dict[str, np.ndarray]:
    """Per-site observables from the raw streams (critmc models.py:325-351).

    e = E / N for all; m2, its root absm and its square m4; Ising also m = M / N;
    Potts m2 = (q sum_k rho_k^2 - 1) / (q - 1) (clipped at 0) and mmax =
    (q max_k rho_k - 1) / (q - 1) with rho = counts / N; O(n) m2 = |M / N|^2.
    """
    n = float(meta["N"])
    kind = meta["model"]
    if kind not in ("ising", "potts", "on"):
        raise ValueError(f"no observables for model kind {kind!r}")
    obs: dict[str, np.ndarray] = {"e": np.asarray(raw["E"], dtype=np.float64) / n}
    if kind == "ising":
        obs["m"] = raw["M"] / n
        m2 = np.square(obs["m"])
    elif kind == "potts":
        q = int(meta["q"])
        rho = raw["counts"] / n
        m2 = np.maximum((q * np.einsum("tk,tk->t", rho, rho) - 1.0) / (q - 1.0), 0.0)
        obs["mmax"] = (q * np.max(rho, axis=1) - 1.0) / (q - 1.0)
    else:
        mvec = raw["M"] / n
        m2 = np.einsum("tk,tk->t", mvec, mvec)
    obs["m2"] = m2
    obs["absm"] = np.sqrt(m2)
    obs["m4"] = np.square(m2)
    return obs
