"""Simulation's host logic against critmc's own (critmc sim.py:134-297).

Both are driven through the same deterministic fake ``advance`` (the fixture
holds critmc's side, made by tests/golden/make_golden.py): the advance calls
(chunk sizes, the schedule with its tuned Wolff count, the Metropolis step),
the tuning reports and the series metadata must agree.  Also the update-string
parser and TimeSeries helpers."""

from __future__ import annotations

import numpy as np
import pytest
from exact_helpers import SIM_SCENARIOS, fake_advance, golden, summarize_series

from critmc_b200 import ON, Ising, Simulation, TimeSeries, parse_updates, square
from critmc_b200.io import to_jsonable


class _Chain:
    def __init__(self, state):
        self.state = np.array(state, copy=True)

    def fetch(self):
        return self.state.copy()


def _fake(kind):
    base = Ising if kind == "ising" else ON
    args = (square(8),) if kind == "ising" else (square(8), 2)

    class Fake(base):
        calls: list = []

        def to_device(self, state, rng, device=None):
            return _Chain(state)

        def advance(self, chain, running, beta, schedule, n_meas):
            Fake.calls.append([int(n_meas), np.asarray(schedule).tolist(), running.get("step")])
            return fake_advance(len(Fake.calls) - 1, schedule, n_meas, self.n_sites, kind)

    Fake.calls = []
    return Fake(*args), Fake


@pytest.mark.parametrize("case", range(len(SIM_SCENARIOS)))
def test_simulation_host_logic_matches_critmc(case):
    kind, updates, therm, n_chunks, n_run, chunk = SIM_SCENARIOS[case]
    ref = golden()["simulation_host_logic"][case]
    model, cls = _fake(kind)
    sim = Simulation(model, 0.5, updates, seed=11)
    tuning = sim.thermalize(therm, n_chunks=n_chunks)
    ts = sim.run(n_run, chunk=chunk)
    got = to_jsonable({"calls": cls.calls, "tuning": tuning, "final_tuning": sim.tuning(),
                       "series": summarize_series(ts.raw, ts.meta), "n_therm": sim.n_therm, "n_meas": sim.n_meas})
    assert got["calls"] == ref["calls"]
    assert got["tuning"] == ref["tuning"] and got["final_tuning"] == ref["final_tuning"]
    assert got["series"] == ref["series"]
    assert (got["n_therm"], got["n_meas"]) == (ref["n_therm"], ref["n_meas"])


def test_update_strings():
    assert parse_updates("heatbath+4*overrelax") == [("heatbath", None), ("overrelax", 4)]
    assert parse_updates(" Metropolis + wolff ") == [("metropolis", None), ("wolff", None)]
    assert parse_updates("sw++2*metropolis") == [("sw", None), ("metropolis", 2)]
    for bad in ("", "+", "0*metropolis", "x*metropolis", "flip"):
        with pytest.raises(ValueError):
            parse_updates(bad)


def test_time_series_helpers():
    raw = {"E": np.arange(6.0), "M": np.arange(6), "aux": np.zeros((6, 4), np.int64)}
    ts = TimeSeries(raw, {"model": "ising", "N": 4, "L": 2, "beta": 0.3, "n_meas": 6})
    assert len(ts) == 6 and ts.beta == 0.3 and ts.n_sites == 4 and ts.L == 2
    np.testing.assert_allclose(ts["e"], raw["E"] / 4)
    assert {"e", "m", "m2", "absm", "E"} <= set(ts.keys())
    with pytest.raises(KeyError):
        ts["nope"]
    parts = [ts.slice(0, 2), ts.slice(2, None)]
    joined = TimeSeries.concatenate(parts)
    np.testing.assert_array_equal(joined.raw["E"], raw["E"])
    assert joined.meta["n_meas"] == 6
    with pytest.raises(ValueError):
        TimeSeries.concatenate([])
