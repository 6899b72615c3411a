"""The C port of critmc's CPU Ising kernel (the benchmark's CPU baseline) equals
critmc bit for bit: its PCG64DXSM against numpy's raw outputs, and whole runs
against seeded critmc ``Simulation`` runs (fixtures that critmc itself wrote,
``tests/golden/make_port_golden.py``)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from critmc_b200 import hypercubic

FIX = json.loads((Path(__file__).resolve().parent / "golden" / "critmc_port.json").read_text())


def _words(state: str, inc: str) -> np.ndarray:
    return oracle.pcg_words({"state": int(state), "inc": int(inc)})


def test_pcg64dxsm_equals_numpy_raw_outputs():
    ref = FIX["pcg_raw"]
    w = _words(ref["state"], ref["inc"])
    got = oracle.pcg_raw(w, 64)
    np.testing.assert_array_equal(got, np.array([int(x) for x in ref["outputs"]], dtype=np.uint64))


@pytest.mark.parametrize("case", FIX["cases"], ids=lambda c: f"{c['shape']}-{c['updates']}")
def test_port_run_equals_critmc(case):
    lat = hypercubic(tuple(case["shape"]))
    s = np.ascontiguousarray(case["start"], dtype=np.int8)
    w = _words(case["pcg_state"], case["pcg_inc"])
    e, m, aux, _ = oracle.critmc_ising_run(s, lat.nbr, w, case["beta"], case["h"], case["schedule"], case["n_meas"])
    np.testing.assert_array_equal(e, case["Eb"])
    np.testing.assert_array_equal(m, case["M"])
    np.testing.assert_array_equal(aux, case["aux"])
    np.testing.assert_array_equal(s, np.asarray(case["final"], dtype=np.int8))
