"""Flat-histogram sampling on the CPU: level mapping and window walk (host
logic), and the oracle's Wang-Landau / multicanonical walks pinned against
exact densities of states (critmc tests/test_flathist.py patterns)."""

from __future__ import annotations

import numpy as np
import pytest
from exact_helpers import JointDOS, ising_log_g_square6, kaufman_energy
from flathist_replay import replay_multicanonical, replay_wang_landau, walk_into_window

from critmc_b200 import Ising, Potts, square
from critmc_b200.flathist import EnergyLevels, MucaResult, WLResult


def test_energy_levels_mapping():
    """critmc tests/test_flathist.py:9-16: 4x4 Ising has 17 levels from -32 to 32,
    E = -24 is level 2, per-site [-2, 0] is levels 0..8; 4x4 q=3 Potts has 33."""
    ising = EnergyLevels.of(Ising(square(4)))
    assert (ising.size, ising.energies[0], ising.energies[-1]) == (17, -32, 32)
    assert ising.index(-24) == 2 and ising.window(-2.0, 0.0) == (0, 8)
    potts = EnergyLevels.of(Potts(square(4), 3))
    assert (potts.size, potts.index(-32)) == (33, 0)
    for bad in (lambda: ising.window(0.5, 0.5), lambda: EnergyLevels.of(Ising(square(4), h=0.1))):
        with pytest.raises(ValueError):
            bad()


@pytest.mark.parametrize("kind", ["ising", "potts"])
def test_walk_into_window_reaches_the_window(kind):
    model = Ising(square(8)) if kind == "ising" else Potts(square(6), 4)
    lv = EnergyLevels.of(model)
    lo, hi = lv.window(*{"ising": (-1.9, -1.6), "potts": (-1.5, -1.2)}[kind])
    gen = np.random.default_rng(5)
    s = model.initial_state("random", gen)
    idx = walk_into_window(model, s, lv, lo, hi, gen)
    assert lo <= idx <= hi and idx == lv.index(model.energy(s))


def _walker(model, seed, window):
    lv = EnergyLevels.of(model)
    gen = np.random.default_rng(seed)
    s = model.initial_state("random", gen)
    idx = walk_into_window(model, s, lv, *window, gen)
    key = gen.integers(0, 1 << 32, size=2, dtype=np.uint64).astype(np.uint32)
    return lv, s.astype(np.int8), idx, key


@pytest.mark.parametrize("one_over_t", [False, True])
def test_oracle_wang_landau_ising_against_exact_dos(one_over_t):
    model = Ising(square(6))
    lv = EnergyLevels.of(model)
    window = (0, lv.size - 1)
    lv, s, idx, key = _walker(model, 3, window)
    r = replay_wang_landau((6, 6), 0, s, key, idx, window, lv.size, 36, 1e-6, one_over_t=one_over_t)
    res = WLResult(lv, r["ln_g"], r["visited"], window, r["trials"], r["ln_f"], 0.0, r["stages"])
    reference = ising_log_g_square6()
    seen = res.visited
    assert (seen == np.isfinite(reference)).all()
    assert np.abs(res.normalized()[seen] - reference[seen]).mean() < {True: 0.02, False: 0.08}[one_over_t]
    kaufman = np.array([kaufman_energy(b, 6) for b in (0.3, 0.44, 0.6)])
    bound = {True: 0.01, False: 0.03}[one_over_t] + 1e-5 * np.abs(kaufman)
    assert (np.abs(res.canonical([0.3, 0.44, 0.6])["u"] - kaufman) <= bound).all()
    assert res.stages[0]["ln_f"] == 1.0


def test_oracle_wang_landau_potts_window():
    model = Potts(square(4, 3), 3)
    jd = JointDOS("potts3_dos_square4x3")
    exact = {float(e): float(np.log(c)) for e, c in zip(jd.energies, jd.counts.sum(axis=1))}
    lv = EnergyLevels.of(model)
    window = lv.window(-2.0, -1.0)
    lv, s, idx, key = _walker(model, 4, window)
    r = replay_wang_landau((4, 3), 3, s, key, idx, window, lv.size, 12, 1e-7)
    res = WLResult(lv, r["ln_g"], r["visited"], window, r["trials"], r["ln_f"], 0.0)
    got = res.normalized()
    e = lv.energies
    diff = got[res.visited] - np.array([exact[x] for x in e[res.visited]])
    assert np.ptp(diff) < 0.02
    assert e[res.visited].max() <= -12


def test_oracle_multicanonical_reweighting_to_canonical():
    model = Ising(square(6))
    lng = ising_log_g_square6()
    lv = EnergyLevels.of(model)
    window = (0, lv.size - 1)
    lv, s, idx, key = _walker(model, 8, window)
    ln_w = np.where(np.isfinite(lng), -lng, -np.inf)
    r = replay_multicanonical((6, 6), 0, s, key, idx, window, ln_w, 36, 200_000, n_therm=100)
    out = MucaResult(lv, lng, r["level_series"], r["order_series"], window, r["hist"])
    assert (out.hist > 0).sum() == np.isfinite(lng).sum()
    for b in (0.3, 0.44, 0.55):
        assert out.canonical(b)["u"][0] == pytest.approx(kaufman_energy(b, 6), abs=0.01)
    # the order series is the magnetisation of the configuration: check the last one
    assert r["order_series"][-1] == int(r["state"].astype(np.int64).sum())


def test_oracle_multicanonical_potts_order_series_and_m2():
    model = Potts(square(4, 2), 3)
    jd = JointDOS("potts3_dos_square4x2")
    lv = EnergyLevels.of(model)
    g = jd.counts.sum(axis=1)
    lng = np.full(lv.size, -np.inf)
    for e, c in zip(jd.energies, g):
        if c > 0:
            lng[lv.index(e)] = np.log(c)
    window = (0, lv.size - 1)
    lv, s, idx, key = _walker(model, 2, window)
    ln_w = np.where(np.isfinite(lng), -lng, -np.inf)
    r = replay_multicanonical((4, 2), 3, s, key, idx, window, ln_w, 8, 100_000)
    out = MucaResult(lv, lng, r["level_series"], r["order_series"], window, r["hist"])
    counts = np.bincount(r["state"].astype(np.int64), minlength=3)
    assert r["order_series"][-1] == int((counts ** 2).sum())
    beta, n = 0.8, 8
    # the fixture's order variable is q sum_k n_k^2
    exact_m2 = jd.average(beta, lambda e, o: (o / n ** 2 - 1.0) / 2.0)
    got = out.canonical(beta)
    assert got["m2"][0] == pytest.approx(exact_m2, abs=0.02)
    assert got["u"][0] == pytest.approx(jd.average(beta, lambda e, o: e) / n, abs=0.02)


@pytest.mark.parametrize("kind,shape,q,win", [("ising", (8, 8), 0, (-1.9, -1.6)), ("potts", (6, 6), 4, (-1.5, -1.2)),
                                              ("ising", (4, 4, 4), 0, (-2.0, -1.5))])
def test_oracle_descent_is_consistent_and_reaches_the_window_from_order(kind, shape, q, win):
    """The oracle's greedy descent (critmc flathist.py:96-130 rule): the final
    level is always the configuration's, with matching M / counts; from a random
    start it may stall above the window (a straight domain wall), from the
    ordered configuration it walks up into the window."""
    from flathist_replay import initial_order

    import oracle
    from critmc_b200 import hypercubic

    model = Ising(hypercubic(shape)) if kind == "ising" else Potts(hypercubic(shape), q)
    lv = EnergyLevels.of(model)
    lo, hi = lv.window(*win)
    rng = np.random.default_rng(9)
    for start in ["random"] * 5 + ["ordered"] * 2:
        s = model.initial_state(start, rng).astype(np.int8)
        order = initial_order(s, q)
        key = rng.integers(0, 1 << 32, size=2, dtype=np.uint64).astype(np.uint32)
        idx, steps = oracle.fh_descend(s, shape, q, key, lv.index(model.energy(s)), order, (lo, hi), 10**6)
        assert idx == lv.index(model.energy(s))
        np.testing.assert_array_equal(order, initial_order(s, q))
        assert (steps >= 0) == (lo <= idx <= hi)
        if start == "ordered":
            assert steps >= 0


def test_oracle_wang_landau_equal_height_point_matches_critmc():
    """The oracle's converged ln g of the q = 10 Potts 8 x 8 torus gives the
    equal-height point that critmc's own Wang-Landau gives (fixture)."""
    from exact_helpers import golden
    from scipy.optimize import brentq
    from scipy.special import logsumexp

    ref = golden()["potts10_L8_equal_height"]
    model = Potts(square(8), 10)
    lv = EnergyLevels.of(model)
    window = lv.window(*ref["window"])
    lv, s, idx, key = _walker(model, 1, (0, lv.size - 1))
    import oracle
    from flathist_replay import initial_order

    idx, steps = oracle.fh_descend(s, (8, 8), 10, key, idx, initial_order(s, 10), window, 10**6)
    assert steps >= 0
    r = replay_wang_landau((8, 8), 10, s, key, idx, window, lv.size, 64, ref["ln_f_final"])
    e = lv.energies / 64
    v = r["visited"]

    def f(b):
        a = np.where(v, r["ln_g"] - b * lv.energies, -np.inf)
        p = np.exp(a - logsumexp(a[v]))
        low = e < ref["split"]
        return np.log(p[low].max()) - np.log(p[~low].max())

    assert brentq(f, 1.2, 1.5) == pytest.approx(ref["beta"], abs=0.002)


def test_analysis_methods_match_critmc_on_a_synthetic_record():
    """MucaResult / WLResult analysis (critmc flathist.py:133-171, 322-452) on a
    seeded synthetic record equals critmc's own methods on it (fixture)."""
    from exact_helpers import golden, synthetic_muca

    ref = golden()["flathist_analysis"]
    ln_g, idx, order, window, hist = synthetic_muca()
    lv = EnergyLevels("potts", 64, 128, 10)
    mu = MucaResult(lv, ln_g, idx, order, window, hist)
    got = mu.canonical([1.36, 1.40, 1.44])
    for k, v in ref["canonical"].items():
        np.testing.assert_allclose(got[k], v, rtol=1e-12)
    np.testing.assert_allclose(mu.order_parameter_m2()[:8], ref["m2_head"], rtol=1e-12)
    assert mu.average(1.40, mu.order_parameter_m2()) == pytest.approx(ref["average_m2"], rel=1e-12)
    for smooth in (0.0, 0.01):
        np.testing.assert_allclose(mu.energy_distribution(1.40, smooth)[1], ref[f"p_smooth{smooth}"],
                                   rtol=1e-10, atol=1e-300)
        for k, v in mu.double_peak(1.40, -1.3, smooth).items():
            assert v == pytest.approx(ref[f"double_peak_smooth{smooth}"][k], rel=1e-10, nan_ok=True), k
        assert mu.equal_height_beta((1.2, 1.6), -1.3, smooth) == pytest.approx(ref[f"equal_height_smooth{smooth}"],
                                                                             abs=1e-9)
    for k, v in mu.double_peak(1.40).items():
        assert v == pytest.approx(ref["double_peak_auto_split"][k], rel=1e-10, nan_ok=True), k
    for k, v in mu.phase_means(1.40, -1.3).items():
        assert v == pytest.approx(ref["phase_means"][k], rel=1e-12), k
    assert mu.equal_weight_beta((1.2, 1.6), -1.3) == pytest.approx(ref["equal_weight"], abs=1e-9)
    visited = hist > 0
    for win, key in ((window, "wl_window"), ((0, lv.size - 1), "wl_full")):
        wl = WLResult(lv, np.where(visited, ln_g, 0.0), visited, win, 0, 0.0, 0.0)
        np.testing.assert_allclose(np.where(visited, wl.normalized(), 0.0), ref[key]["normalized"], rtol=1e-12)
        got = wl.canonical([1.36, 1.40])
        for k, v in ref[key]["canonical"].items():
            np.testing.assert_allclose(got[k], v, rtol=1e-10)


def _with_oracle_walkers(monkeypatch):
    import fake_walkers

    import critmc_b200.flathist as fh

    monkeypatch.setattr(fh, "_Walkers", fake_walkers.OracleWalkers)
    return fh


def _start(walkers, w):
    return walkers.spins[w].numpy().copy(), int(walkers.idx[w]), walkers.keys[w].numpy().view(np.uint32).copy()


def test_wang_landau_schedule_on_the_cpu_equals_the_replay(monkeypatch):
    """WangLandau.run's host schedule (critmc flathist.py:247-320), driven through
    oracle-backed walkers: every walker of a batch equals the replay of its run."""
    fh = _with_oracle_walkers(monkeypatch)
    model = Potts(square(4, 3), 3)
    wins = [None, (-2.0, -1.0), (-1.5, -0.5)]
    wl = fh.WangLandau(model, e_window=wins, n_walkers=3, seed=2)
    starts = [_start(wl.walkers, w) for w in range(3)]
    results = wl.run(1e-3, checkpoints=[500, 20_000, 10**9])
    for w, res in enumerate(results):
        s, idx, key = starts[w]
        r = replay_wang_landau((4, 3), 3, s, key, idx, wl.windows[w], res.levels.size, 12, 1e-3,
                               checkpoints=[500, 20_000, 10**9])
        assert np.array_equal(res.ln_g, r["ln_g"]) and np.array_equal(res.visited, r["visited"])
        assert res.trials == r["trials"] and res.ln_f == r["ln_f"] and res.stages == r["stages"]
        assert [c[0] for c in res.checkpoints] == [c[0] for c in r["checkpoints"]]
        for a, b in zip(res.checkpoints, r["checkpoints"]):
            assert a[1] == b[1] and np.array_equal(a[2], b[2])
    np.testing.assert_array_equal(wl.walkers.window.numpy(), np.array(wl.windows))


def test_multicanonical_run_on_the_cpu_equals_the_replay(monkeypatch):
    fh = _with_oracle_walkers(monkeypatch)
    model = Ising(square(6))
    lng = ising_log_g_square6()
    mu = fh.Multicanonical(model, lng, seed=8, n_walkers=2)
    starts = [_start(mu.walkers, w) for w in range(2)]
    outs = mu.run(500, sweeps_per_meas=2, n_therm=20)
    for w, o in enumerate(outs):
        s, idx, key = starts[w]
        r = replay_multicanonical((6, 6), 0, s, key, idx, mu.window, mu.ln_w, 72, 500, n_therm=20)
        np.testing.assert_array_equal(o.level_series, r["level_series"])
        np.testing.assert_array_equal(o.order_series, r["order_series"])
        np.testing.assert_array_equal(o.hist, r["hist"])
