"""Chains on byte lattices (int8 Ising for sizes outside the multi-spin-coded
layout, q-state Potts), advanced by ``critmc_ising_byte_run`` /
``critmc_potts_run`` (one thread block per chain)."""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import ptr, require_cuda, stream_handle, to_dev, to_host
from .layout import cb_pack, cb_unpack

N_AUX = 4


class _ByteChain:
    def __init__(self, model, state: np.ndarray, key: np.ndarray, device):
        self.device = require_cuda(device)
        self.model = model
        self.shape = tuple(model.lattice.shape)
        self.dims = self.shape + (1,) * (3 - len(self.shape))
        self.key = np.ascontiguousarray(key, dtype=np.uint32).reshape(1, 2)
        self.spins = to_dev(cb_pack(np.asarray(state, dtype=np.int8), self.shape), self.device)
        self.sweep = 0

    def fetch(self) -> np.ndarray:
        return cb_unpack(to_host(self.spins), self.shape)


class IsingByteChain(_ByteChain):
    """Ising chain with one int8 per site (any even extents)."""

    def advance(self, running, beta, schedule, n_meas):
        dev = self.device
        tables, _ = self.model.tables(beta)
        sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
        run = torch.tensor([[running["e_b"], running["m"]]], dtype=torch.int64, device=dev)
        e = torch.empty((1, n_meas), dtype=torch.int64, device=dev)
        m = torch.empty((1, n_meas), dtype=torch.int64, device=dev)
        aux = torch.empty((1, n_meas, N_AUX), dtype=torch.int64, device=dev)
        lx, ly, lz = self.dims
        _lib.call_on(dev, "critmc_ising_byte_run", ptr(self.spins), len(self.shape), lx, ly, lz, 1,
                     self.key.ctypes.data, tables.ctypes.data, 1, self.sweep, sched.ctypes.data, len(sched), n_meas,
                     ptr(run), ptr(e), ptr(m), ptr(aux), stream_handle(dev))
        self.sweep += int(sched[:, 1].sum()) * n_meas
        r = to_host(run)[0]
        running["e_b"], running["m"] = int(r[0]), int(r[1])
        e_b = to_host(e)[0]
        mm = to_host(m)[0]
        h = self.model.h
        energy = e_b - h * mm if h != 0.0 else e_b
        return {"E": energy, "Eb": e_b, "M": mm, "aux": to_host(aux)[0]}


class PottsChain(_ByteChain):
    """q-state Potts chain, states 0..q-1 in int8."""

    def advance(self, running, beta, schedule, n_meas):
        dev = self.device
        q = self.model.q
        sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
        betas = np.array([beta], dtype=np.float64)
        energy = torch.tensor([running["energy"]], dtype=torch.int64, device=dev)
        counts = torch.from_numpy(np.asarray(running["counts"], dtype=np.int64).reshape(1, q)).to(dev)
        e = torch.empty((1, n_meas), dtype=torch.int64, device=dev)
        co = torch.empty((1, n_meas, q), dtype=torch.int64, device=dev)
        aux = torch.empty((1, n_meas, N_AUX), dtype=torch.int64, device=dev)
        lx, ly, lz = self.dims
        _lib.call_on(dev, "critmc_potts_run", ptr(self.spins), len(self.shape), lx, ly, lz, q, 1,
                     self.key.ctypes.data, betas.ctypes.data, 1, self.sweep, sched.ctypes.data, len(sched), n_meas,
                     ptr(energy), ptr(counts), ptr(e), ptr(co), ptr(aux), stream_handle(dev))
        self.sweep += int(sched[:, 1].sum()) * n_meas
        running["energy"] = int(to_host(energy)[0])
        running["counts"] = to_host(counts)[0].copy()
        return {"E": to_host(e)[0], "counts": to_host(co)[0], "aux": to_host(aux)[0]}
