"""Serving: each request's result is the same served in a mix (sliced into
ticks, batched with other requests, admitted late) as run alone through the
per-model entry point in one call."""

from __future__ import annotations

import numpy as np
import pytest

from critmc_b200.serve import Request, Server, open_chain

pytestmark = pytest.mark.gpu

REQUESTS = [
    Request("ising", 16, 0.44, 900, seed=1),  # byte lattice item
    Request("ising", 64, 0.4406868, 1200, seed=2),  # multi-spin-coded item
    Request("ising", 512, 0.45, 300, seed=3),  # multi-block lane
    Request("ising", 128, 0.3, 700, seed=4, h=0.2, updates="heatbath"),
    Request("ising", 8, 0.2216546, 500, seed=5, dim=3, updates="2*metropolis+heatbath"),
    Request("potts", 32, 1.42, 800, seed=6, q=10),
    Request("potts", 16, 1.0, 600, seed=7, q=3, updates="heatbath"),
    Request("xy", 32, 1.1, 400, seed=8, updates="heatbath+2*overrelax"),
    Request("heisenberg", 16, 0.7, 300, seed=9, updates="metropolis+overrelax"),
    Request("xy", 64, 1.0, 250, seed=10),
    Request("ising", 256, 0.46, 400, seed=11),
    Request("ising", 512, 0.40, 260, seed=12),
    Request("ising", 512, 0.47, 180, seed=13, updates="heatbath"),
    Request("ising", 512, 0.43, 90, seed=14),
]


def _alone(req: Request, cuda):
    model, chain, running = open_chain(req, cuda)
    raw = model.advance(chain, running, req.beta, req.schedule(), req.sweeps)
    return raw, chain.fetch()


def _check(res, cuda):
    raw, state = _alone(res.request, cuda)
    for k, v in raw.items():
        np.testing.assert_array_equal(res.series[k], v, err_msg=f"{res.request} {k}")
    np.testing.assert_array_equal(res.state, state)


@pytest.mark.parametrize("team_after_s", [None, 2e-3])
def test_served_results_equal_alone(cuda, team_after_s):
    """team_after_s 2 ms: the longer requests run as thread-block-cluster teams."""
    srv = Server(cuda, tick_ms=0.5, keep_state=True, team_after_s=team_after_s)
    reqs = []
    for i, r in enumerate(REQUESTS):
        reqs.append(Request(**{**r.__dict__, "arrival": 0.004 * i, "rid": i}))
    results = srv.run(reqs)
    assert len(results) == len(REQUESTS)
    st = srv.stats()
    assert st["ticks"] > 3  # the requests were sliced and overlapped
    if team_after_s is not None:
        assert len(srv.team_sizes_used) > 1, srv.team_sizes_used
    for res in results:
        assert res.finished >= res.admitted >= res.arrival
        _check(res, cuda)


def test_admission_waits_for_hbm(cuda):
    """With room for about one L=512 lattice the others queue, then run."""
    reqs = [Request("ising", 512, 0.44, 120, seed=20 + i, rid=i, arrival=0.0) for i in range(3)]
    reqs.append(Request("potts", 16, 1.3, 200, seed=30, rid=3, arrival=0.0))
    budget = Server.request_bytes(reqs[0]) + Server.request_bytes(reqs[3]) + 10
    srv = Server(cuda, tick_ms=0.5, hbm_budget=budget, keep_state=True)
    results = srv.run(reqs)
    st = srv.stats()
    assert st["peak_hbm_bytes"] <= budget
    assert st["max_queued"] >= 1
    assert sorted(r.request.rid for r in results) == [0, 1, 2, 3]
    adm = sorted(r.admitted for r in results if r.request.model == "ising")
    assert adm[1] > adm[0] and adm[2] > adm[1]
    for res in results:
        _check(res, cuda)


def test_summary_mode_error_bars(cuda):
    from exact_helpers import gamma_error

    req = Request("ising", 64, 0.44, 3000, seed=50, rid=0, arrival=0.0)
    srv = Server(cuda, tick_ms=0.3, keep_series=False, stats_lag=128)
    (res,) = srv.run([req])
    raw, _ = _alone(req, cuda)
    st = res.stats["Eb"]
    mean, err, tau = gamma_error(raw["Eb"].astype(np.float64))
    assert st["n"] == 3000 and st["mean"] == pytest.approx(mean, rel=1e-12)
    if not st["truncated"]:
        assert st["error"] == pytest.approx(err, rel=1e-7)


def test_summary_mode_sums_match(cuda):
    reqs = [Request("ising", 32, 0.44, 300, seed=40, rid=0, arrival=0.0),
            Request("potts", 16, 1.4, 250, seed=41, rid=1, arrival=0.0)]
    srv = Server(cuda, tick_ms=0.3, keep_series=False)
    for res in srv.run(reqs):
        raw, _ = _alone(res.request, cuda)
        for k, v in res.series.items():
            want = np.asarray(raw[k]).reshape(res.request.sweeps, -1).sum(axis=0)
            np.testing.assert_array_equal(v, want)
