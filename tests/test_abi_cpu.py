"""The C ABI library loads without a GPU and exports every declared entry point."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from critmc_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "critmc_b200.h"


def declared() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(critmc_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    names = declared()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_the_header():
    assert set(declared()) <= set(_lib.SIGNATURES), set(declared()) - set(_lib.SIGNATURES)


def test_version_and_error_text():
    L = _lib.lib()
    assert L.critmc_version() >= 100
    kind = np.zeros(16, np.uint32)
    thr = np.zeros(16, np.uint32)
    st = L.critmc_ising_class_table(9, 4, 0.4, 0.0, kind.ctypes.data, thr.ctypes.data, None)
    assert st == -3
    assert "metropolis and heatbath" in _lib.last_error()


def test_invalid_arguments_fail_before_any_launch():
    """Validation runs on the host: no GPU is touched for bad arguments."""
    L = _lib.lib()
    sched = np.array([[0, 1]], np.int64)
    keys = np.zeros(2, np.uint32)
    tables = np.zeros(64, np.uint32)
    # odd extent
    st = L.critmc_ising_byte_run(None, 2, 5, 4, 1, 1, keys.ctypes.data, tables.ctypes.data, 1, 0,
                                 sched.ctypes.data, 1, 1, None, None, None, None, None)
    assert st in (-1, -3)
    # lx not a multiple of 64 for the MSC layout
    st = L.critmc_ising_msc_run(None, 2, 96, 4, 1, 1, keys.ctypes.data, tables.ctypes.data, 1, 0,
                                sched.ctypes.data, 1, 1, None, None, None, None, None, 0, 8, None)
    assert st == -3 and "64" in _lib.last_error()
    # cluster move in a schedule
    bad = np.array([[3, 1]], np.int64)
    dummy = ctypes.c_void_p(16)
    st = L.critmc_potts_run(dummy, 2, 4, 4, 1, 3, 1, keys.ctypes.data,
                            np.array([1.0]).ctypes.data, 1, 0, bad.ctypes.data, 1, 1, dummy, dummy,
                            dummy, dummy, dummy, None)
    assert st == -3


def test_flat_histogram_and_on_cluster_arguments_fail_before_any_launch():
    L = _lib.lib()
    d = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    keys = np.zeros(2, np.uint32)
    # mode 2 does not exist
    st = L.critmc_fh_run(2, d, 2, 4, 4, 1, 0, 1, d, 9, d, d, d, d, d, d, d, d, d, d, 10, 1, None, None, None)
    assert st == -1 and "mode" in _lib.last_error()
    # Potts q out of range, and more than 2^24 sites per walker
    st = L.critmc_fh_run(0, d, 2, 4, 4, 1, 200, 1, d, 9, d, d, d, d, d, d, d, d, d, d, 10, 1, None, None, None)
    assert st == -1
    st = L.critmc_fh_run(0, d, 2, 8192, 4096, 1, 0, 1, d, 9, d, d, d, d, d, d, d, d, d, d, 10, 1, None, None, None)
    assert st == -1 and "2^24" in _lib.last_error()
    # Wang-Landau without its per-walker ln f arrays; multicanonical without outputs
    st = L.critmc_fh_run(0, d, 2, 4, 4, 1, 0, 1, d, 9, d, d, d, d, d, d, None, d, d, d, 10, 1, None, None, None)
    assert st == -1 and "ln_f" in _lib.last_error()
    st = L.critmc_fh_run(1, d, 2, 4, 4, 1, 0, 1, d, 9, d, d, d, d, d, d, None, None, None, None, 10, 3, None,
                         None, None)
    assert st == -1 and "idx_out" in _lib.last_error()
    # O(n) cluster moves: n = 4, an unknown algorithm, a negative beta
    st = L.critmc_on_cluster_update(d, 2, 4, 4, 1, 4, 1, keys.ctypes.data, 1.0, 3, 0, d, d, None)
    assert st == -3
    st = L.critmc_on_cluster_update(d, 2, 4, 4, 1, 2, 1, keys.ctypes.data, 1.0, 0, 0, d, d, None)
    assert st == -1 and "wolff" in _lib.last_error()
    st = L.critmc_on_cluster_update(d, 2, 4, 4, 1, 2, 1, keys.ctypes.data, -1.0, 4, 0, d, d, None)
    assert st == -1 and "beta" in _lib.last_error()


@pytest.mark.parametrize("beta", [0.0, 0.44, 3.0])
def test_potts_tables_are_monotone(beta):
    b = np.zeros(8, np.uint64)
    w = np.zeros(8, np.uint64)
    _lib.call("critmc_potts_tables", 4, beta, b.ctypes.data, w.ctypes.data)
    assert b[0] == 1 << 32
    assert np.all(np.diff(b[:5].astype(np.float64)) <= 0)
    assert w[4] == 1 << 52 if beta > 0 else True


def test_item_struct_matches_the_header():
    """The ctypes mirror has the C struct's size; item preparation is host-only."""
    from critmc_b200.items import ITEM_ON, ITEM_POTTS, CritmcItem

    lib = _lib.lib()
    assert ctypes.sizeof(CritmcItem) == lib.critmc_items_buffer_bytes(1) - lib.critmc_items_buffer_bytes(0)
    it = CritmcItem()
    it.kind, it.dim, it.lx, it.ly, it.n_rows = 0, 2, 64, 64, 1
    it.codes[0], it.reps[0] = 0, 1
    assert _lib.lib().critmc_item_prepare(ctypes.byref(it), 0.4406868, 0.0, 1.0) == 0
    assert it.kind_tab[0][0] != 0 or it.thr_tab[0][0] != 0
    it.kind, it.q_or_n = ITEM_POTTS, 3
    assert _lib.lib().critmc_item_prepare(ctypes.byref(it), 1.0, 0.0, 1.0) == 0
    assert it.boltz[0] != 0
    it.kind, it.q_or_n, it.codes[0] = ITEM_ON, 2, 5
    assert _lib.lib().critmc_item_prepare(ctypes.byref(it), 1.25, 0.0, 0.5) == 0
    assert (it.beta, it.step) == (1.25, 0.5)
    it.kind = ITEM_POTTS  # over-relaxation is an O(n) move only
    assert _lib.lib().critmc_item_prepare(ctypes.byref(it), 1.0, 0.0, 1.0) != 0
    it.kind = 9
    assert _lib.lib().critmc_item_prepare(ctypes.byref(it), 1.0, 0.0, 1.0) != 0
    assert _lib.lib().critmc_run_items(None, 0, None, 0, None, 0, None) == 0


def test_item_team_sizes_are_checked_before_any_device_work():
    """A team of 2, 4, 8 or 16 blocks is a thread-block cluster; other sizes are refused."""
    from critmc_b200.items import TEAM_SIZES, CritmcItem, ItemRun

    assert TEAM_SIZES == (1, 2, 4, 8, 16)
    lib = _lib.lib()
    it = CritmcItem()
    it.kind, it.dim, it.lx, it.ly, it.n_rows = 0, 2, 64, 64, 1
    it.codes[0], it.reps[0] = 0, 1
    it.team = 3
    buf = ctypes.create_string_buffer(int(lib.critmc_items_buffer_bytes(1)))
    st = lib.critmc_run_items(ctypes.byref(it), 1, ctypes.cast(buf, ctypes.c_void_p), len(buf), None, 0, None)
    assert st == -1  # CRITMC_ERR_INVALID
    assert "team" in _lib.last_error()
    with pytest.raises(ValueError, match="team"):
        ItemRun(None, None, {}, 0.4, np.array([[0, 1]]), 1, team=5)
    assert lib.critmc_items_team_clusters(0, 0, 2, 3) == -1  # refused before any device call
    assert lib.critmc_items_team_clusters(9, 0, 2, 8) == -1
