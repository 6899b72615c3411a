"""Real runs of the bounds-checked flavour (-DCRITMC_CHECK) see no bad index.

A child process loads ``libcritmc_b200_check.so`` (CRITMC_B200_CHECK=1) and runs
multi-spin-coded Ising, byte-lattice Ising and Potts, and O(n) chains, each
checked bit for bit against the oracle, then asks the library for its record
of out-of-range indices: there must be none.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import oracle
from critmc_b200 import ON, Ising, Potts, _lib, hypercubic, square
from critmc_b200.on_models import ONChain
assert _lib.lib()._name.endswith("libcritmc_b200_check.so"), _lib.lib()._name
rng = np.random.default_rng(3)
for shape, sched in (((128, 6), [[0, 1], [2, 1]]), ((64, 4, 6), [[0, 1]]), ((18, 10), [[0, 1]])):
    model = Ising(hypercubic(shape))
    s0 = model.initial_state("random", rng)
    key = np.array([7, 9], np.uint32)
    ch = model.to_device(s0, np.random.default_rng(0), "cuda")
    ch.key = key.reshape(ch.key.shape)
    raw = model.advance(ch, model.begin(s0), 0.44, np.array(sched), 5)
    ref = s0.copy()
    run = oracle.ising_msc_run if ch.__class__.__name__ == "_IsingMscChain" else oracle.ising_byte_run
    e, m, aux, _ = run(ref, shape, key, 0.44, 0.0, sched, 5)
    assert np.array_equal(raw["Eb"], e) and np.array_equal(ch.fetch(), ref), shape
pm = Potts(square(16), 5)
p0 = pm.initial_state("random", rng)
pc = pm.to_device(p0, np.random.default_rng(1), "cuda")
pm.advance(pc, pm.begin(p0), 1.1, np.array([[0, 1], [2, 1]]), 4)
om = ON(square(16), 3)
o0 = om.initial_state("random", rng).astype(np.float32)
oc = ONChain(om, o0, np.array([3, 4], np.uint32), "cuda", lane="block")
oc.advance({"step": 1.0}, 0.8, np.array([[2, 1], [5, 2]]), 3)
buf = ctypes.create_string_buffer(1024)
hits = _lib.lib().critmc_check_report(buf, 1024)
print("bad indices:", hits, buf.value.decode())
assert hits == 0, buf.value.decode()
"""


def test_checked_flavour_sees_no_bad_index(tmp_path):
    from critmc_b200 import _build

    _build.build(check=True)
    env = dict(os.environ, CRITMC_B200_CHECK="1")
    res = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], env=env, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "bad indices: 0" in res.stdout
