"""Work items: many chains of any model and size advanced by one call.

``critmc_run_items`` (``include/critmc_b200.h``) takes a list of
``critmc_item`` descriptors, one per chain slice, and runs them with a
persistent kernel per model family whose blocks pull items from a queue.
``ItemRun`` builds the descriptors for chain objects of this package
(multi-spin-coded Ising, byte Ising, Potts, O(n)), allocates the outputs and
returns the same raw dictionaries as ``Model.advance``.  Results equal the
per-model entry points bit for bit: the random streams are indexed by chain
key, sweep and site only.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .byte_models import IsingByteChain, PottsChain
from .device import empty_bytes, ptr, stream_handle, to_host
from .models import _IsingMscChain
from .on_models import ONChain

ITEM_MSC_ISING, ITEM_BYTE_ISING, ITEM_POTTS, ITEM_ON = 0, 1, 2, 3


class CritmcItem(ctypes.Structure):
    """Mirror of ``critmc_item`` in include/critmc_b200.h."""

    _fields_ = [
        ("spins", ctypes.c_void_p),
        ("running", ctypes.c_void_p),
        ("counts", ctypes.c_void_p),
        ("e_out", ctypes.c_void_p),
        ("vec_out", ctypes.c_void_p),
        ("sc_out", ctypes.c_void_p),
        ("ss_out", ctypes.c_void_p),
        ("aux_out", ctypes.c_void_p),
        ("kind", ctypes.c_int32),
        ("dim", ctypes.c_int32),
        ("lx", ctypes.c_int32),
        ("ly", ctypes.c_int32),
        ("lz", ctypes.c_int32),
        ("q_or_n", ctypes.c_int32),
        ("key", ctypes.c_uint32 * 2),
        ("sweep0", ctypes.c_uint32),
        ("n_meas", ctypes.c_int32),
        ("n_rows", ctypes.c_int32),
        ("codes", ctypes.c_int32 * 4),
        ("reps", ctypes.c_int32 * 4),
        ("rule", ctypes.c_int32 * 2),
        ("beta", ctypes.c_float),
        ("step", ctypes.c_float),
        ("kind_tab", (ctypes.c_uint32 * 16) * 2),
        ("thr_tab", (ctypes.c_uint32 * 16) * 2),
        ("boltz", ctypes.c_uint64 * 8),
        ("weight", ctypes.c_uint64 * 8),
        ("team", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


TEAM_SIZES = (1, 2, 4, 8, 16)


class ItemRun:
    """One slice of work for one chain: ``n_meas`` applications of ``schedule``.

    ``team``: thread blocks advancing the chain together (1; or 2, 4, 8, 16 as a
    thread-block cluster, for large lattices); the results do not depend on it.
    The run owns the device buffers that ``item`` points to (outputs, running
    sums): keep it alive until the launch has completed.
    """

    def __init__(self, model, chain, running: dict, beta: float, schedule: np.ndarray, n_meas: int,
                 team: int = 1):
        if team not in TEAM_SIZES:
            raise ValueError(f"team must be one of {TEAM_SIZES}, got {team}")
        self.model, self.chain, self.running = model, chain, running
        self.beta = float(beta)
        self.schedule = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
        self.n_meas = int(n_meas)
        dev = chain.device
        shape = tuple(chain.shape)
        dims = shape + (1,) * (3 - len(shape))
        it = CritmcItem()
        it.spins = ptr(chain.words if isinstance(chain, _IsingMscChain) else chain.spins)
        it.dim, (it.lx, it.ly, it.lz) = len(shape), dims
        it.key[0], it.key[1] = int(chain.key.ravel()[0]), int(chain.key.ravel()[1])
        it.sweep0 = chain.sweep
        it.n_meas = self.n_meas
        it.team = int(team)
        it.n_rows = len(self.schedule)
        if it.n_rows > 4:
            raise ValueError("work items take at most 4 schedule rows")
        for r, (code, reps) in enumerate(self.schedule):
            it.codes[r], it.reps[r] = int(code), int(reps)
        n = self.n_meas
        self._t = {}
        if isinstance(chain, (_IsingMscChain, IsingByteChain)):
            it.kind = ITEM_MSC_ISING if isinstance(chain, _IsingMscChain) else ITEM_BYTE_ISING
            self._t["running"] = torch.tensor([running["e_b"], running["m"]], dtype=torch.int64, device=dev)
            self._t["e"] = torch.empty(n, dtype=torch.int64, device=dev)
            self._t["v"] = torch.empty(n, dtype=torch.int64, device=dev)
            h = model.h
        elif isinstance(chain, PottsChain):
            it.kind = ITEM_POTTS
            it.q_or_n = model.q
            self._t["running"] = torch.tensor([running["energy"]], dtype=torch.int64, device=dev)
            self._t["counts"] = torch.from_numpy(np.asarray(running["counts"], dtype=np.int64)).to(dev)
            self._t["e"] = torch.empty(n, dtype=torch.int64, device=dev)
            self._t["v"] = torch.empty((n, model.q), dtype=torch.int64, device=dev)
            h = 0.0
        elif isinstance(chain, ONChain):
            it.kind = ITEM_ON
            it.q_or_n = model.n
            dim = len(shape)
            self._t["e"] = torch.empty(n, dtype=torch.float64, device=dev)
            self._t["v"] = torch.empty((n, model.n), dtype=torch.float64, device=dev)
            self._t["sc"] = torch.empty((n, dim), dtype=torch.float64, device=dev)
            self._t["ss"] = torch.empty((n, dim), dtype=torch.float64, device=dev)
            h = 0.0
        else:
            raise TypeError(f"no work-item form for {type(chain).__name__}")
        self._t["aux"] = torch.empty((n, 4), dtype=torch.int64, device=dev)
        it.running = ptr(self._t.get("running"))
        it.counts = ptr(self._t.get("counts"))
        it.e_out = ptr(self._t["e"])
        it.vec_out = ptr(self._t["v"])
        it.sc_out = ptr(self._t.get("sc"))
        it.ss_out = ptr(self._t.get("ss"))
        it.aux_out = ptr(self._t["aux"])
        _lib.call("critmc_item_prepare", ctypes.byref(it), self.beta, float(h),
                  float(running.get("step", 1.0)))
        self.item = it

    def finish(self) -> dict[str, np.ndarray]:
        """Read the results back (after the run), update the chain's counters."""
        chain, running, t = self.chain, self.running, self._t
        chain.sweep += int(self.schedule[:, 1].sum()) * self.n_meas
        aux = to_host(t["aux"])
        if isinstance(chain, (_IsingMscChain, IsingByteChain)):
            r = to_host(t["running"])
            running["e_b"], running["m"] = int(r[0]), int(r[1])
            e_b, m = to_host(t["e"]), to_host(t["v"])
            h = self.model.h
            return {"E": e_b - h * m if h != 0.0 else e_b, "Eb": e_b, "M": m, "aux": aux}
        if isinstance(chain, PottsChain):
            running["energy"] = int(to_host(t["running"])[0])
            running["counts"] = to_host(t["counts"]).copy()
            return {"E": to_host(t["e"]), "counts": to_host(t["v"]), "aux": aux}
        return {"E": to_host(t["e"]), "M": to_host(t["v"]), "stiff_c": to_host(t["sc"]),
                "stiff_s": to_host(t["ss"]), "aux": aux}


def team_clusters(kind: int, q_or_n: int, dim: int, team: int, device) -> int:
    """Teams of ``team`` blocks of the item kernel for ``kind`` items that the
    GPU runs at once; 0 if it cannot schedule clusters of that size."""
    st = _lib.lib().critmc_items_team_clusters
    with torch.cuda.device(device):
        n = st(int(kind), int(q_or_n), int(dim), int(team))
    if n < 0:
        _lib.check(n)
    return int(n)


def launch_items(items, device, buffer: torch.Tensor | None, *, staging: torch.Tensor | None = None,
                 smem_limit: int = 0, stream=None, control=None) -> torch.Tensor:
    """Run a ctypes array (or list) of ``CritmcItem``; returns the (grown) descriptor buffer.

    ``staging``: pinned host bytes for the asynchronous descriptor copy (see
    ``critmc_run_items``); ``None`` copies from pageable memory.  ``control``:
    an armed ``RunControl`` bounding the launch (None: runs to completion).
    """
    n = len(items)
    if n == 0:
        return buffer
    arr = items if isinstance(items, ctypes.Array) else (CritmcItem * n)(*items)
    need = _lib.lib().critmc_items_buffer_bytes(n)
    if buffer is None or buffer.numel() < need:
        buffer = empty_bytes(need, device)
    if staging is not None and staging.numel() < n * ctypes.sizeof(CritmcItem):
        raise ValueError("staging buffer too small")
    st = stream if stream is not None else stream_handle(device)
    _lib.call_on(device, "critmc_run_items_ctl", ctypes.cast(arr, ctypes.c_void_p), n, ptr(buffer), int(need),
                 staging.data_ptr() if staging is not None else None, int(smem_limit),
                 control.handle if control is not None else None, st)
    return buffer


def run_items(runs: list[ItemRun], device, *, smem_limit: int = 0, buffer: torch.Tensor | None = None,
              stream=None, control=None) -> torch.Tensor:
    """Launch all ``runs`` in one call; returns the descriptor buffer (reuse it).

    ``control``: an armed ``RunControl`` bounding the launch (see ``critmc_b200.control``)."""
    return launch_items([r.item for r in runs], device, buffer, smem_limit=smem_limit, stream=stream,
                        control=control)
