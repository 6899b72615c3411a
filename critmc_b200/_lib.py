"""ctypes binding of ``libcritmc_b200.so`` (the C ABI in ``include/critmc_b200.h``).

The library is built in-tree by :mod:`critmc_b200._build`.  Loading fails
loudly when it is missing: there is no CPU fallback for any sampler.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libcritmc_b200.so"
# CRITMC_B200_CHECK=1 loads the bounds-checked flavour (built on first use)
LIB_CHECK_PATH = PKG / "libcritmc_b200_check.so"

_lib: ctypes.CDLL | None = None

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_U32 = ctypes.c_uint32
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> (restype, argtypes); kept in the order of include/critmc_b200.h
SIGNATURES: dict[str, tuple] = {
    "critmc_version": (_I32, []),
    "critmc_last_error": (_I32, [_P, _I32]),
    "critmc_check_report": (_I64, [_P, _I32]),
    "critmc_ising_class_table": (_I32, [_I32, _I32, _D, _D, _P, _P, _P]),
    "critmc_ising_msc_scratch_bytes": (_I64, [_I32, _I32]),
    "critmc_ising_msc_run": (
        _I32,
        [_P, _I32, _I32, _I32, _I32, _I32, _P, _P, _I32, _U32, _P, _I32, _I32, _P, _P, _P, _P, _P,
         _I32, _I32, _P],
    ),
    "critmc_ising_msc_batch_scratch_bytes": (_I64, [_I32, _I32]),
    "critmc_ising_msc_run_batch": (_I32, [_P, _I32, _I32, _I32, _I32, _I32, _P, _I32, _P, _I32, _I32, _P, _I32,
                                          _P]),
    "critmc_ising_msc_measure": (_I32, [_P, _I32, _I32, _I32, _I32, _I32, _P, _P]),
    "critmc_item_prepare": (_I32, [_P, _D, _D, _D]),
    "critmc_items_buffer_bytes": (_I64, [_I32]),
    "critmc_items_team_clusters": (_I32, [_I32, _I32, _I32, _I32]),
    "critmc_run_items": (_I32, [_P, _I32, _P, _I64, _P, _I32, _P]),
    "critmc_ising_msc_noalloc_max_scratch_bytes": (_I64, []),
    "critmc_ising_msc_run_noalloc": (
        _I32,
        [_P, _I32, _I32, _I32, _I32, _I32, _P, _P, _I32, _U32, _P, _I32, _I32, _P, _P, _P, _P, _I32,
         _P],
    ),
    "critmc_ising_msc_init": (_I32, [_P, _I32, _I32, _I32, _I32, _I32, _P, _I32, _P]),
    "critmc_ising_byte_run": (
        _I32,
        [_P, _I32, _I32, _I32, _I32, _I32, _P, _P, _I32, _U32, _P, _I32, _I32, _P, _P, _P, _P, _P],
    ),
    "critmc_potts_run": (
        _I32,
        [_P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P, _I32, _U32, _P, _I32, _I32, _P, _P, _P, _P,
         _P, _P],
    ),
    "critmc_potts_tables": (_I32, [_I32, _D, _P, _P]),
    "critmc_pt_swap_table": (_I32, [_I32, _P, _I32, _P]),
    "critmc_ea_coupling_bits": (_I32, [_I32, _I32, _I32, _I32, _P, _P]),
    "critmc_ea_pt_run": (
        _I32,
        [_P, _P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P, _P, _I32, _P, _P, _U32, _I32, _I32, _I32,
         _P, _P, _P, _P, _P, _P],
    ),
    "critmc_on_run": (
        _I32,
        [_P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P, _P, _I32, _U32, _P, _I32, _I32, _P, _P, _P,
         _P, _P, _P],
    ),
    "critmc_on_grid_scratch_bytes": (_I64, [_I32, _I32, _I32, _I32]),
    "critmc_graph_cache_set_capacity": (_I32, [_I32]),
    "critmc_cluster_scratch_bytes": (_I64, [_I32, _I64]),
    "critmc_stream_state_bytes": (_I64, [_I32, _I32]),
    "critmc_fh_run": (_I32, [_I32, _P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _I32, _P, _P, _P, _P, _P, _P, _P,
                             _P, _P, _P, _I64, _I32, _P, _P, _P]),
    "critmc_fh_descend": (_I32, [_P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _I32, _P, _P, _P, _I64, _P, _P]),
    "critmc_stream_update": (_I32, [_P, _I32, _I32, _I32, _I64, _P, _I32, _P]),
    "critmc_cluster_update": (
        _I32, [_I32, _P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _D, _I32, _U32, _P, _P, _P, _P, _P]),
    "critmc_on_cluster_update": (_I32, [_P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _D, _I32, _U32, _P, _P, _P]),
    "critmc_chain_create": (_I32, [_I32, _P, _I32, _D, _U32, _U32, ctypes.c_uint64, _I32, _P, _P]),
    "critmc_chain_destroy": (_I32, [_P]),
    "critmc_chain_info": (_I32, [_P, _P, _P, _P]),
    "critmc_chain_set_step": (_I32, [_P, _D]),
    "critmc_advance": (_I32, [_P, _D, _P, _I32, _I32, _P, _P, _P, _P, _P]),
    "critmc_get_state": (_I32, [_P, _P, _P, _P]),
    "critmc_set_state": (_I32, [_P, _P, _P]),
    "critmc_batch_create": (_I32, [_P]),
    "critmc_batch_destroy": (_I32, [_P]),
    "critmc_batch_submit": (_I32, [_P, _P, _D, _P, _I32, _I32, _P, _P, _P, _P, _P]),
    "critmc_batch_poll": (_I32, [_P, _P, _P, _I32, _P]),
    "critmc_batch_cancel": (_I32, [_P, ctypes.c_int64]),
    "critmc_batch_pending": (_I32, [_P]),
    "critmc_control_create": (_I32, [_P]),
    "critmc_control_destroy": (_I32, [_P]),
    "critmc_control_arm": (_I32, [_P, _I64]),
    "critmc_control_cancel": (_I32, [_P]),
    "critmc_control_status": (_I32, [_P]),
    "critmc_control_wait": (_I32, [_P, _P]),
    "critmc_ea_campaign_run_ctl": (
        _I32, [_P, _I32, _I32, _I32, _P, _P, _I32, _U32, _I32, _I32, _I32, _P, _I64, _P, _P, _P]),
    "critmc_run_items_ctl": (_I32, [_P, _I32, _P, _I64, _P, _I32, _P, _P]),
    "critmc_ea_campaign_buffer_bytes": (_I64, [_I32, _I64]),
    "critmc_ea_campaign_run": (
        _I32, [_P, _I32, _I32, _I32, _P, _P, _I32, _U32, _I32, _I32, _I32, _P, _I64, _P, _P]),
    "critmc_graph_cache_size": (_I32, []),
    "critmc_on_run_grid": (
        _I32,
        [_P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P, _P, _I32, _U32, _P, _I32, _I32, _P, _P, _P,
         _P, _P, _P, _I32, _P],
    ),
}


class CritmcError(RuntimeError):
    """Error status returned by the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(f"critmc_b200 error {status}: {message}")
        self.status = status


def lib() -> ctypes.CDLL:
    """Load the shared library (once)."""
    global _lib
    if _lib is None:
        check = os.environ.get("CRITMC_B200_CHECK", "") not in ("", "0")
        path = LIB_CHECK_PATH if check else LIB_PATH
        if not path.exists():
            if os.environ.get("CRITMC_B200_NO_BUILD"):
                raise RuntimeError(f"{path} is missing; build it with python -m critmc_b200._build"
                                   + (" --check" if check else ""))
            from . import _build

            _build.build(check=check)
        L = ctypes.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    lib().critmc_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != 0:
        raise CritmcError(status, last_error())


def call(name: str, *args) -> int:
    """Call ``name`` and raise :class:`CritmcError` on a non-zero status."""
    status = getattr(lib(), name)(*args)
    check(status)
    return status


# Entry points that only fill host tables: they touch no device and need no guard.
HOST_ONLY = frozenset({
    "critmc_version", "critmc_last_error", "critmc_ising_class_table", "critmc_ising_msc_scratch_bytes",
    "critmc_item_prepare", "critmc_items_buffer_bytes", "critmc_ising_msc_noalloc_max_scratch_bytes",
    "critmc_potts_tables", "critmc_pt_swap_table", "critmc_ea_coupling_bits", "critmc_on_grid_scratch_bytes",
    "critmc_graph_cache_set_capacity", "critmc_cluster_scratch_bytes", "critmc_stream_state_bytes",
    "critmc_ea_campaign_buffer_bytes", "critmc_graph_cache_size",
    "critmc_control_arm", "critmc_control_cancel", "critmc_control_status",
    "critmc_ising_msc_batch_scratch_bytes",
})


def call_on(device, name: str, *args) -> int:
    """Call ``name`` with ``device`` made current for the duration of the call.

    The C entry points launch on the calling thread's current CUDA device
    (``cudaGetDevice``); buffers and the stream handle that a wrapper passes
    belong to the wrapper's own device.  Without this guard a chain on cuda:1,
    driven from a thread whose current device is 0, would launch on GPU 0
    against GPU 1's memory.
    """
    import torch

    with torch.cuda.device(device):
        return call(name, *args)
