"""Host-side serving logic: the workload generator and request bookkeeping."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from critmc_b200.serve import DEFAULT_UPDATES, Request, Server, mixed_workload


def test_workload_is_seeded_and_has_the_stated_mix():
    a = mixed_workload(3000, 200.0, seed=3)
    b = mixed_workload(3000, 200.0, seed=3)
    assert [r.__dict__ for r in a] == [r.__dict__ for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert abs(arr[-1] / len(a) - 1 / 200.0) < 0.1 / 200.0  # mean gap 1/rate
    kinds = {k: [r for r in a if r.model == k] for k in ("ising", "potts", "xy")}
    for k, rs in kinds.items():
        assert abs(len(rs) / len(a) - 1 / 3) < 0.04, k
    assert {r.L for r in kinds["ising"]} == {16, 32, 64, 128, 256, 512, 1024}
    assert {r.L for r in kinds["potts"]} == {16, 32, 64, 128}
    assert {r.L for r in kinds["xy"]} == {32, 64, 128}
    assert all(0.38 <= r.beta <= 0.50 for r in kinds["ising"])
    assert all(1.35 <= r.beta <= 1.50 and r.q == 10 for r in kinds["potts"])
    assert all(0.8 <= 1 / r.beta <= 1.0 for r in kinds["xy"])
    sw = np.log10([r.sweeps for r in a])
    assert sw.min() >= 3 - 1e-9 and sw.max() <= 5 + 1e-9
    assert abs(sw.mean() - 4.0) < 0.05
    assert len({r.seed for r in a}) == len(a)


def test_request_schedules_and_sizes():
    r = Request("xy", 32, 1.0, 10, updates="heatbath+4*overrelax")
    np.testing.assert_array_equal(r.schedule(), [[2, 1], [5, 4]])
    assert Request("potts", 16, 1.0, 1).schedule().tolist() == [[0, 1]]
    assert set(DEFAULT_UPDATES) == {"ising", "potts", "xy", "heisenberg"}
    assert Server.request_bytes(Request("ising", 1024, 0.4, 1)) == 1024 * 1024 // 8 + 4096
    assert Server.request_bytes(Request("ising", 32, 0.4, 1)) == 32 * 32 + 4096
    assert Server.request_bytes(Request("xy", 64, 1.0, 1)) == 64 * 64 * 8 + 4096


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error")
def test_server_needs_a_gpu():
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        Server()


def test_team_choice_follows_the_cost_model():
    """_team_for: one block when that is predicted within team_after_s; else the
    smallest team predicted within it; else the smallest within TEAM_SLACK of
    the fastest.  Exercised on an object with the server's policy fields only
    (no device)."""
    from critmc_b200.serve import COSTS, TEAM_SLACK, TEAMS

    class Policy:
        _team_for = Server._team_for

        def __init__(self, after, max_team=8):
            self.team_after_s, self.teams = after, tuple(t for t in TEAMS if t <= max_team)
            self.costs = dict(COSTS)

        def _team_fits(self, req, family, team):  # every size schedulable (no device here)
            return True

    big = Request("ising", 1024, 0.44, 100_000)
    small = Request("ising", 16, 0.44, 100_000)
    assert Policy(None)._team_for(big, "msc") == 1
    assert Policy(1.0)._team_for(small, "msc") == 1  # one block already fast enough
    p = Policy(1.0)
    per = big.sweeps
    pred = {t: per * (p.costs[(f"team{t}", "msc")][0] + p.costs[(f"team{t}", "msc")][1] * big.n_sites)
            for t in p.teams}
    t = p._team_for(big, "msc")
    within = [u for u in p.teams if pred[u] <= 1.0]
    if within:
        assert t == within[0]
    else:
        best = min(pred.values())
        assert pred[t] <= TEAM_SLACK * best and all(pred[u] > TEAM_SLACK * best for u in p.teams if u < t)
    assert Policy(1.0, max_team=4)._team_for(big, "msc") <= 4
    # a generous threshold keeps long requests on one block
    assert Policy(1e9)._team_for(big, "msc") == 1
