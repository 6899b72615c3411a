"""CPU tests: the oracle's RNG and tables, the layouts, the library's host code."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from critmc_b200 import Ising, square, cubic
from critmc_b200 import layout

# Random123 known-answer vectors for Philox4x32-10 (counter, key) -> output
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expected", KAT)
def test_oracle_philox_known_answers(ctr, key, expected):
    assert tuple(int(v) for v in oracle.philox(ctr, key)) == expected


def test_msc_layout_round_trip():
    rng = np.random.default_rng(1)
    for shape in [(64, 2), (128, 6), (64, 4, 2), (256, 10)]:
        n = int(np.prod(shape))
        s = (2 * rng.integers(0, 2, n) - 1).astype(np.int8)
        w = layout.msc_pack(s, shape)
        assert w.shape == (2, int(np.prod(shape[1:])), shape[0] // 64)
        np.testing.assert_array_equal(layout.msc_unpack(w, shape), s)


def test_checkerboard_order_is_colour_consistent():
    shape = (8, 6, 4)
    lat = cubic(4)
    order = layout.checkerboard_order(shape)
    coords = np.stack(np.unravel_index(order.ravel(), shape, order="F"), 1).reshape(2, -1, 3)
    for c in range(2):
        assert np.all(coords[c].sum(axis=1) % 2 == c)
    assert sorted(order.ravel()) == list(range(int(np.prod(shape))))
    assert lat.bipartite


def test_oracle_bond_energy_matches_numpy():
    rng = np.random.default_rng(3)
    for L, dim in ((64, 2), (8, 3)):
        lat = square(L) if dim == 2 else cubic(L)
        s = (2 * rng.integers(0, 2, lat.n_sites) - 1).astype(np.int8)
        assert oracle.ising_bond_energy(s, lat.shape) == Ising(lat).bond_energy(s)


@pytest.mark.parametrize("algo", [0, 2])
@pytest.mark.parametrize("h", [0.0, 0.37])
def test_library_class_table_matches_oracle(algo, h):
    from critmc_b200 import _lib

    for z in (2, 4, 6):
        for beta in (0.05, 0.4406868, 1.3):
            kind = np.zeros(16, np.uint32)
            thr = np.zeros(16, np.uint32)
            dep = ctypes.c_int32(-1)
            _lib.call("critmc_ising_class_table", algo, z, beta, h, kind.ctypes.data,
                      thr.ctypes.data, ctypes.byref(dep))
            ref = oracle.ising_table(algo, z, beta, h)
            np.testing.assert_array_equal(kind, ref[0])
            np.testing.assert_array_equal(thr, ref[1])
            assert dep.value == int(algo == 0 and h != 0.0)


def test_oracle_metropolis_bookkeeping_is_exact():
    """Incremental E_b/M of the replay equal a recomputation (critmc test_kernels.py:39-40)."""
    lat = square(64, 4)
    rng = np.random.default_rng(5)
    s = (2 * rng.integers(0, 2, lat.n_sites) - 1).astype(np.int8)
    e, m, aux, running = oracle.ising_msc_run(s, lat.shape, (7, 9), 0.44, 0.2,
                                              [[0, 1], [2, 2]], 20)
    assert running[0] == Ising(lat).bond_energy(s)
    assert running[1] == int(s.astype(np.int64).sum())
    assert e[-1] == running[0] and m[-1] == running[1]
    assert np.all(aux[:, 0] > 0)
