"""The series file format (critmc io.py:33-48): a file written by critmc itself
(fixture from tests/golden/make_golden.py) loads here, and saving it again
gives the same archive members, dtypes and metadata text."""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from critmc_b200.io import META_MEMBER, load_npz, save_npz, to_jsonable
from critmc_b200.sim import TimeSeries

FIXTURE = Path(__file__).resolve().parent / "golden" / "critmc_series_ising4.npz"


def test_a_critmc_series_loads_and_derives():
    ts = TimeSeries.load(FIXTURE)
    assert set(ts.raw) == {"E", "Eb", "M", "aux"}
    assert ts.raw["E"].dtype == np.int64 and ts.raw["aux"].shape == (200, 4)
    assert ts.meta["model"] == "ising" and ts.meta["N"] == 16 and ts.meta["n_meas"] == 200
    assert ts.meta["mean_cluster"] == "nan"  # a non-finite float is stored as its text
    np.testing.assert_allclose(ts["e"], ts.raw["E"] / 16.0)
    np.testing.assert_allclose(ts["m2"], (ts.raw["M"] / 16.0) ** 2)


def test_saving_again_gives_the_same_archive(tmp_path):
    ts = TimeSeries.load(FIXTURE)
    out = ts.save(tmp_path / "again.npz")
    with np.load(FIXTURE) as a, np.load(out) as b:
        assert a.files == b.files
        for name in a.files:
            assert a[name].dtype == b[name].dtype and a[name].shape == b[name].shape
            np.testing.assert_array_equal(a[name], b[name])
        assert str(a[META_MEMBER]) == str(b[META_MEMBER])


def test_json_conventions_and_reserved_name(tmp_path):
    meta = {1: (np.int64(3), np.float64(0.5)), "p": Path("/x/y"), "bad": math.inf, "arr": np.arange(3)}
    assert to_jsonable(meta) == {"1": [3, 0.5], "p": "/x/y", "bad": "inf", "arr": [0, 1, 2]}
    assert math.isnan(to_jsonable(np.float64("nan")))  # numpy scalars stay numbers
    with pytest.raises(ValueError):
        save_npz(tmp_path / "x.npz", {META_MEMBER: np.zeros(2)}, {})
    p = save_npz(tmp_path / "sub" / "y", {"a": np.arange(4)}, {"k": (1, 2)})
    arrays, m = load_npz(str(p) + ".npz" if not str(p).endswith(".npz") else p)
    np.testing.assert_array_equal(arrays["a"], np.arange(4))
    assert m == {"k": [1, 2]}
