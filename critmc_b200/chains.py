"""Chains owned by the library: a Python view of the handle ABI.

``Chain`` wraps ``critmc_chain_create`` / ``critmc_advance`` /
``critmc_get_state`` / ``critmc_set_state``: the library keeps the lattice,
running sums, Philox key and sweep counter on the device, and the caller
passes states in critmc's site order.  ``Batch`` wraps the batch queue
(``critmc_batch_submit`` / ``poll`` / ``cancel``), which runs the submissions
of many chains together as work items.  ``advance`` returns the raw series of
critmc's ``Model.advance`` (src/critmc/models.py:58-68).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .device import ptr, require_cuda, stream_handle, to_host
from .models import UPDATE_CODES
from .sim import parse_updates

KINDS = {"ising": 0, "potts": 1, "on": 2}
STARTS = {"random": 0, "ordered": 1, "state": 2}


def schedule_array(updates) -> np.ndarray:
    if isinstance(updates, str):
        rows = parse_updates(updates)
        return np.array([[UPDATE_CODES[n], 1 if k is None else k] for n, k in rows], dtype=np.int64)
    return np.ascontiguousarray(updates, dtype=np.int64).reshape(-1, 2)


class Chain:
    """One chain held by the library (``critmc_chain``)."""

    def __init__(self, kind: str, shape, *, q_or_n: int = 0, h: float = 0.0, seed: int = 0, chain_id: int = 0,
                 start: str = "random", state: np.ndarray | None = None, device=None):
        self.device = require_cuda(device)
        self.kind = kind
        self.shape = tuple(int(v) for v in shape)
        self.q_or_n = int(q_or_n)
        self.n_sites = int(np.prod(self.shape))
        dims = (ctypes.c_int32 * 3)(*(self.shape + (0, 0, 0))[:3])
        handle = ctypes.c_void_p()
        init = None
        if state is not None:
            start = "state"
            init = self._host_state(state)
        _lib.call_on(self.device, "critmc_chain_create", KINDS[kind], dims, self.q_or_n, float(h), seed & 0xFFFFFFFF,
                     (seed >> 32) & 0xFFFFFFFF, int(chain_id), STARTS[start],
                     init.ctypes.data if init is not None else None, ctypes.byref(handle))
        self._h = handle

    def _host_state(self, state) -> np.ndarray:
        if self.kind == "on":
            return np.ascontiguousarray(state, dtype=np.float64).reshape(self.n_sites, self.q_or_n)
        return np.ascontiguousarray(state, dtype=np.int8).reshape(self.n_sites)

    def info(self) -> dict:
        layout, sweep, key = ctypes.c_int32(), ctypes.c_uint32(), (ctypes.c_uint32 * 2)()
        _lib.call_on(self.device, "critmc_chain_info", self._h, ctypes.byref(layout), ctypes.byref(sweep), key)
        return {"layout": ("msc", "byte", "float")[layout.value], "sweep": sweep.value,
                "key": np.array(list(key), dtype=np.uint32)}

    def set_step(self, step: float) -> None:
        _lib.call_on(self.device, "critmc_chain_set_step", self._h, float(step))

    def outputs(self, n_meas: int) -> dict[str, torch.Tensor]:
        dev, n = self.device, n_meas
        out = {"aux": torch.empty((n, 4), dtype=torch.int64, device=dev)}
        if self.kind == "on":
            dim = len(self.shape)
            out["f64"] = torch.empty(n * (1 + self.q_or_n + 2 * dim), dtype=torch.float64, device=dev)
        else:
            out["e"] = torch.empty(n, dtype=torch.int64, device=dev)
            out["m"] = torch.empty((n, self.q_or_n) if self.kind == "potts" else n, dtype=torch.int64, device=dev)
        return out

    def raw(self, out: dict, n_meas: int) -> dict[str, np.ndarray]:
        """Model.advance's raw dictionary from the device outputs."""
        aux = to_host(out["aux"])
        if self.kind == "on":
            f = to_host(out["f64"])
            n, dim, q = n_meas, len(self.shape), self.q_or_n
            return {"E": f[:n], "M": f[n:n + n * q].reshape(n, q),
                    "stiff_c": f[n + n * q:n + n * q + n * dim].reshape(n, dim),
                    "stiff_s": f[n + n * q + n * dim:].reshape(n, dim), "aux": aux}
        if self.kind == "potts":
            return {"E": to_host(out["e"]), "counts": to_host(out["m"]), "aux": aux}
        return {"Eb": to_host(out["e"]), "M": to_host(out["m"]), "aux": aux}

    def advance(self, beta: float, updates, n_meas: int) -> dict[str, np.ndarray]:
        sched = schedule_array(updates)
        out = self.outputs(n_meas)
        _lib.call_on(self.device, "critmc_advance", self._h, float(beta), sched.ctypes.data, len(sched), int(n_meas),
                     ptr(out.get("e")), ptr(out.get("m")), ptr(out["aux"]), ptr(out.get("f64")),
                     stream_handle(self.device))
        return self.raw(out, n_meas)

    def state(self) -> tuple[np.ndarray, np.ndarray | None]:
        """(configuration in critmc's site order, running sums or None)."""
        if self.kind == "on":
            s = np.empty((self.n_sites, self.q_or_n), dtype=np.float64)
            run = None
        else:
            s = np.empty(self.n_sites, dtype=np.int8)
            run = np.empty(2 if self.kind == "ising" else 1 + self.q_or_n, dtype=np.int64)
        _lib.call_on(self.device, "critmc_get_state", self._h, s.ctypes.data,
                     run.ctypes.data if run is not None else None, stream_handle(self.device))
        return s, run

    def set_state(self, state) -> None:
        s = self._host_state(state)
        _lib.call_on(self.device, "critmc_set_state", self._h, s.ctypes.data, stream_handle(self.device))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().critmc_chain_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Batch queue over library-held chains (``critmc_batch``)."""

    def __init__(self, device=None):
        self.device = require_cuda(device)
        handle = ctypes.c_void_p()
        _lib.call_on(self.device, "critmc_batch_create", ctypes.byref(handle))
        self._h = handle
        self._subs: dict[int, tuple] = {}

    def submit(self, chain: Chain, beta: float, updates, n_meas: int) -> int:
        sched = schedule_array(updates)
        out = chain.outputs(n_meas)
        ticket = ctypes.c_int64()
        _lib.call_on(self.device, "critmc_batch_submit", self._h, chain._h, float(beta), sched.ctypes.data,
                     len(sched), int(n_meas), ptr(out.get("e")), ptr(out.get("m")), ptr(out["aux"]),
                     ptr(out.get("f64")), ctypes.byref(ticket))
        self._subs[ticket.value] = (chain, out, n_meas)
        return ticket.value

    def cancel(self, ticket: int) -> None:
        _lib.call_on(self.device, "critmc_batch_cancel", self._h, int(ticket))
        self._subs.pop(ticket, None)

    def pending(self) -> int:
        return _lib.lib().critmc_batch_pending(self._h)

    def poll(self, max_done: int = 1 << 20) -> dict[int, dict[str, np.ndarray]]:
        """Run every pending submission; returns {ticket: raw series}."""
        n = min(max_done, max(1, len(self._subs)))
        done = (ctypes.c_int64 * n)()
        n_done = ctypes.c_int32()
        _lib.call_on(self.device, "critmc_batch_poll", self._h, stream_handle(self.device), done, n,
                     ctypes.byref(n_done))
        res = {}
        for t in list(done)[:n_done.value]:
            chain, out, n_meas = self._subs.pop(t)
            res[t] = chain.raw(out, n_meas)
        return res

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().critmc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
