"""The split evaluation of the acceptance-plane stream equals plain Philox4x32-10.

The multi-spin-coded kernels evaluate the uniform part of the plane stream once
per launch and only the per-word part per word (``philox.h``); the stream
definition, which the CPU oracle replays, is the plain call.  Checked here on
the host for random keys, sweeps, colours and words, with both plane groups,
at the default round count and with explicit 10 and 7 rounds.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "critmc_b200" / "csrc"


@pytest.mark.parametrize("rounds", [0, 10, 7])
def test_split_plane_stream_equals_philox(tmp_path, rounds):
    """rounds 0: the library's default functions; 10 and 7: the explicit-round variants."""
    so = tmp_path / f"libplanes{rounds}.so"
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", f"-I{CSRC}",
                    str(HERE / "plane_stream_harness.c"), "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    rng = np.random.default_rng(rounds)
    n, groups = 20000, 2
    rows = rng.integers(0, 2**32, (n, 5), dtype=np.uint64).astype(np.uint32)
    rows[:, 3] &= 1  # colour
    rows[:1000, 4] = np.arange(1000)  # small word indices
    rows[1000:2000, 2] = 0xFFFFFFFF  # last sweep of the counter range
    plain = np.zeros((n, groups, 4), np.uint32)
    split = np.zeros_like(plain)
    lib.plane_eval(ctypes.c_int(n), ctypes.c_int(groups), ctypes.c_int(rounds), ctypes.c_void_p(rows.ctypes.data),
                   ctypes.c_void_p(plain.ctypes.data), ctypes.c_void_p(split.ctypes.data))
    np.testing.assert_array_equal(split, plain)
    assert len(np.unique(plain[:, 0, 0])) > n * 0.99


@pytest.mark.parametrize("rounds", [10, 7])
def test_header_philox_equals_the_oracles_independent_one(tmp_path, rounds):
    """The library header's Philox and the oracle's independent implementation agree at the
    round counts the library uses (10 everywhere; 7 for the optional acceptance planes)."""
    import oracle

    so = tmp_path / "libphilox.so"
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", f"-I{CSRC}", str(HERE / "plane_stream_harness.c"),
                    "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    rng = np.random.default_rng(100 + rounds)
    n = 3000
    rows = rng.integers(0, 2**32, (n, 6), dtype=np.uint64).astype(np.uint32)
    got = np.zeros((n, 4), np.uint32)
    lib.philox_eval(ctypes.c_int(n), ctypes.c_int(rounds), ctypes.c_void_p(rows.ctypes.data),
                    ctypes.c_void_p(got.ctypes.data))
    want = np.stack([oracle.philox_rounds(r[:4], r[4:], rounds) for r in rows])
    np.testing.assert_array_equal(got, want)
