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


def test_double_exp_within_two_ulp(tmp_path):
    out = tmp_path / "libcmd.so"
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", f"-I{CSRC}",
                    str(HERE / "fpmath_harness.c"), "-o", str(out), "-lm"], check=True)
    lib = ctypes.CDLL(str(out))
    lib.cm_eval_d.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    x = np.concatenate([rng.uniform(-745, 709, 200_000), rng.uniform(-1, 1, 200_000),
                        rng.uniform(-40, 0, 200_000), [0.0, -1e-300, 709.0, -744.0]])
    o = np.zeros_like(x)
    lib.cm_eval_d(x.ctypes.data, o.ctypes.data, len(x))
    exact = np.exp(x)
    normal = exact > 2.3e-308
    err = np.abs(o[normal] - exact[normal]) / np.spacing(exact[normal])
    assert err.max() <= 2.0
    assert np.all(np.abs(o[~normal] - exact[~normal]) <= 2 * np.spacing(0.0) + 1e-300)


def test_double_log_within_two_ulp(tmp_path):
    out = tmp_path / "libcml.so"
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", f"-I{CSRC}",
                    str(HERE / "fpmath_harness.c"), "-o", str(out), "-lm"], check=True)
    lib = ctypes.CDLL(str(out))
    lib.cm_eval_log_d.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    # the flat-histogram acceptance takes logs of 53-bit uniforms k 2^-53
    u = rng.integers(1, 1 << 53, 300_000, dtype=np.int64).astype(np.float64) * 2.0 ** -53
    x = np.concatenate([u, np.exp(rng.uniform(-700, 700, 200_000)), rng.uniform(0.5, 2.0, 200_000),
                        [2.0 ** -53, 1.0 - 2.0 ** -53, 1.0, 2.0, 5e-324, 1e-310, 1.7e308]])
    o = np.zeros_like(x)
    lib.cm_eval_log_d(x.ctypes.data, o.ctypes.data, len(x))
    exact = np.log(x)
    err = np.abs(o - exact) / np.spacing(np.abs(exact))
    assert err[exact != 0].max() <= 2.0
    assert o[x == 1.0][0] == 0.0
    z = np.array([0.0, -1.0, np.inf])
    oz = np.zeros(3)
    lib.cm_eval_log_d(z.ctypes.data, oz.ctypes.data, 3)
    assert oz[0] == -np.inf and np.isnan(oz[1]) and oz[2] == np.inf
