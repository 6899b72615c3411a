"""Accuracy of the shared single-precision functions (critmc_b200/csrc/fpmath.h)
against double-precision libm, on the host."""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "critmc_b200" / "csrc"


@pytest.fixture(scope="module")
def cm(tmp_path_factory):
    out = tmp_path_factory.mktemp("fpmath") / "libcm.so"
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", f"-I{CSRC}",
                    str(HERE / "fpmath_harness.c"), "-o", str(out), "-lm"], check=True)
    lib = ctypes.CDLL(str(out))
    lib.cm_eval.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_int]

    def ev(which, x, y=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, dtype=np.float32)
        o = np.zeros_like(x)
        lib.cm_eval(which, x.ctypes.data, y.ctypes.data, o.ctypes.data, len(x))
        return o
    return ev


def ulp_err(got: np.ndarray, exact: np.ndarray) -> float:
    exact32 = exact.astype(np.float32)
    ulp = np.spacing(np.abs(exact32)).astype(np.float64)
    return float(np.max(np.abs(got.astype(np.float64) - exact) / ulp))


rng = np.random.default_rng(0)


def test_exp(cm):
    x = np.concatenate([rng.uniform(-87, 88, 200_000), rng.uniform(-2, 2, 200_000)]).astype(np.float32)
    assert ulp_err(cm(0, x), np.exp(x.astype(np.float64))) <= 2.0


def test_log(cm):
    x = np.concatenate([np.exp(rng.uniform(-80, 80, 200_000)), rng.uniform(0.5, 2, 200_000),
                        (np.arange(1, 1 << 12) * 2.0 ** -24)]).astype(np.float32)
    got = cm(1, x)
    ex = np.log(x.astype(np.float64))
    err = np.abs(got - ex)
    # absolute accuracy near 1 (where log -> 0), relative elsewhere
    assert np.all(err <= 3 * np.spacing(np.maximum(np.abs(ex), 1e-7).astype(np.float32)) + 1e-7)


@pytest.mark.parametrize("which,fn", [(2, np.sin), (3, np.cos)])
def test_sincos(cm, which, fn):
    x = rng.uniform(-20, 20, 400_000).astype(np.float32)
    got = cm(which, x)
    assert np.max(np.abs(got - fn(x.astype(np.float64)))) <= 2.5e-7


def test_atan2_and_acos(cm):
    y = rng.standard_normal(400_000).astype(np.float32)
    x = rng.standard_normal(400_000).astype(np.float32)
    got = cm(4, x, y)
    assert np.max(np.abs(got - np.arctan2(y.astype(np.float64), x.astype(np.float64)))) <= 5e-7
    c = rng.uniform(-1, 1, 400_000).astype(np.float32)
    assert np.max(np.abs(cm(5, c) - np.arccos(c.astype(np.float64)))) <= 1e-6
    assert cm(5, np.array([1.0, -1.0], np.float32)).tolist() == pytest.approx([0.0, np.pi], abs=1e-6)
