"""Bounded runs of the persistent kernels: a time budget and a host cancel word.

``RunControl`` wraps a ``critmc_control``: a page of pinned host memory mapped
into the device, with a cancel word that the host sets and a status word that
the kernels set.  Passed to ``MultiSizeCampaign.launch`` / ``run`` or
``items.launch_items``, it makes every thread block of the persistent kernel
poll, between steps or measurements, its own elapsed device time against the
budget and (at most every 100 us) the cancel word.  A block that must stop
records the reason; every block leaves at its next poll, so the kernel returns
by itself and the device stays usable.  critmc has no counterpart: its numba
kernels always run to completion.

A run that stopped leaves its outputs and device state part-way (samples or
items at different steps): restore what was saved before the call.
"""

from __future__ import annotations

import ctypes

from . import _lib
from .device import require_cuda, stream_handle

OK = 0
TIMEOUT = -4    # CRITMC_ERR_TIMEOUT
CANCELLED = -5  # CRITMC_ERR_CANCELLED


class RunStopped(RuntimeError):
    """A bounded run ran out of its budget or was cancelled; its outputs are incomplete."""

    def __init__(self, status: int):
        reason = {TIMEOUT: "ran out of its time budget", CANCELLED: "was cancelled"}.get(status, f"stopped ({status})")
        super().__init__(f"the bounded run {reason}; its outputs are incomplete")
        self.status = status


class RunControl:
    """Cancel word and per-block time budget for the persistent kernels."""

    def __init__(self, device=None):
        self.device = require_cuda(device)
        handle = ctypes.c_void_p()
        _lib.call_on(self.device, "critmc_control_create", ctypes.byref(handle))
        self._h = handle

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def arm(self, budget_s: float | None = None) -> "RunControl":
        """Clear the cancel and status words and set the budget (seconds; None = unbounded).

        Call it only while no run that uses this control is in flight."""
        ns = 0 if budget_s is None else max(1, int(round(budget_s * 1e9)))
        _lib.call("critmc_control_arm", self._h, ns)
        return self

    def cancel(self) -> None:
        """Ask the runs in flight to stop (safe from any host thread)."""
        _lib.call("critmc_control_cancel", self._h)

    def status(self) -> int:
        """0 while nothing stopped, else TIMEOUT or CANCELLED."""
        return int(_lib.lib().critmc_control_status(self._h))

    def wait(self, stream=None, *, raise_on_stop: bool = False) -> int:
        """Synchronise the stream (default: the device's current stream) and return the status."""
        st = int(_lib.lib().critmc_control_wait(self._h, stream if stream is not None else stream_handle(self.device)))
        if st not in (OK, TIMEOUT, CANCELLED):
            _lib.check(st)
        if raise_on_stop and st != OK:
            raise RunStopped(st)
        return st

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().critmc_control_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
