"""Flat-histogram walkers on the GPU: the kernel bit-identical to the oracle
for every model and mode, the Wang-Landau and multicanonical drivers
bit-identical to the CPU replay of their schedules, and critmc's own
statistical checks (critmc tests/test_flathist.py)."""

from __future__ import annotations

import zlib

import numpy as np
import pytest
import torch
from exact_helpers import JointDOS, ising_log_g_square6, kaufman_energy
from flathist_replay import initial_order, replay_multicanonical, replay_wang_landau, walk_into_window

import oracle
from critmc_b200 import Ising, Potts, hypercubic, square
from critmc_b200 import _lib
from critmc_b200.device import ptr, stream_handle
from critmc_b200.flathist import EnergyLevels, Multicanonical, WangLandau

pytestmark = pytest.mark.gpu

KERNEL_CASES = [
    ("ising", (6, 6), 0),
    ("ising", (4, 4, 4), 0),
    ("ising", (16,), 0),
    ("ising", (10, 6), 0),
    ("potts", (4, 3), 3),
    ("potts", (8, 8), 10),
    ("potts", (4, 2, 2), 4),
]


def _model(kind, shape, q):
    lat = hypercubic(shape)
    return Ising(lat) if kind == "ising" else Potts(lat, q)


@pytest.mark.parametrize("path", ["shared", "global"])
@pytest.mark.parametrize("mode", ["wl", "wl_1t", "muca"])
@pytest.mark.parametrize("kind,shape,q", KERNEL_CASES)
def test_fh_kernel_bit_identical_to_oracle(cuda, kind, shape, q, mode, path):
    model = _model(kind, shape, q)
    lv = EnergyLevels.of(model)
    n = model.n_sites
    rng = np.random.default_rng(zlib.crc32(repr((kind, shape, mode)).encode()))
    mid = lv.size // 2
    windows = [(0, lv.size - 1), (max(0, mid - 4), min(lv.size - 1, mid + 3)), (1, lv.size - 2)]
    W = len(windows)
    states, idxs, orders = [], [], []
    for lo, hi in windows:
        s = model.initial_state("random", rng)
        idxs.append(walk_into_window(model, s, lv, lo, hi, rng))
        states.append(s.astype(np.int8))
        orders.append(initial_order(s, q))
    keys = rng.integers(0, 1 << 32, size=(W, 2), dtype=np.uint64).astype(np.uint32)
    lng = rng.normal(0.0, 2.0, size=(W, lv.size))
    if mode == "muca":
        lng[:, 0] = -np.inf  # a forbidden level
    hist = rng.integers(0, 5, size=(W, lv.size)).astype(np.int64)
    ln_f = np.array([0.5, 0.125, 1e-3])
    n_lev = np.array([float(hi - lo + 1) for lo, hi in windows])
    one_t = np.full(W, 1 if mode == "wl_1t" else 0, dtype=np.int32)
    t_base = np.array([0, 3, 7], dtype=np.uint64)
    trials = t_base.copy()
    # device copies
    d = dict(spins=torch.from_numpy(np.stack(states)).to(cuda), keys=torch.from_numpy(keys.view(np.int32)).to(cuda),
             idx=torch.tensor(idxs, dtype=torch.int64, device=cuda),
             order=torch.from_numpy(np.concatenate(orders)).to(cuda), lng=torch.from_numpy(lng.copy()).to(cuda),
             hist=torch.from_numpy(hist.copy()).to(cuda),
             window=torch.tensor(np.array(windows, dtype=np.int32), device=cuda),
             trials=torch.from_numpy(trials.view(np.int64).copy()).to(cuda),
             ln_f=torch.from_numpy(ln_f).to(cuda), n_lev=torch.from_numpy(n_lev).to(cuda),
             one_t=torch.from_numpy(one_t).to(cuda), t_base=torch.from_numpy(t_base.view(np.int64)).to(cuda))
    is_muca = mode == "muca"
    moves, n_meas = (3 * n, 7) if is_muca else (40 * n, 1)
    lx, ly, lz = tuple(shape) + (1,) * (3 - len(shape))
    ref = [dict(s=states[w].copy(), order=orders[w].copy(), lng=lng[w].copy(), hist=hist[w].copy(),
                idx=idxs[w], trials=int(trials[w])) for w in range(W)]
    for block in range(2):
        io = torch.zeros((W, n_meas), dtype=torch.int64, device=cuda) if is_muca else None
        oo = torch.zeros_like(io) if is_muca else None
        flags = 0x10 if path == "global" else 0x20
        _lib.call("critmc_fh_run", int(is_muca) | flags, ptr(d["spins"]), len(shape), lx, ly, lz, q, W, ptr(d["keys"]),
                  lv.size, ptr(d["idx"]), ptr(d["order"]), ptr(d["lng"]), ptr(d["hist"]), ptr(d["window"]),
                  ptr(d["trials"]), ptr(d["ln_f"]), ptr(d["n_lev"]), ptr(d["one_t"]), ptr(d["t_base"]), moves,
                  n_meas, ptr(io), ptr(oo), stream_handle(cuda))
        torch.cuda.synchronize()
        for w in range(W):
            r = ref[w]
            r["idx"], r["trials"], r_io, r_oo = oracle.fh_run(
                int(is_muca), r["s"], shape, q, keys[w], r["idx"], r["order"], r["lng"], r["hist"], windows[w],
                r["trials"], ln_f[w], n_lev[w], bool(one_t[w]), int(t_base[w]), moves, n_meas)
            if is_muca:
                np.testing.assert_array_equal(io[w].cpu().numpy(), r_io)
                np.testing.assert_array_equal(oo[w].cpu().numpy(), r_oo)
        np.testing.assert_array_equal(d["spins"].cpu().numpy(), np.stack([r["s"] for r in ref]))
        np.testing.assert_array_equal(d["idx"].cpu().numpy(), [r["idx"] for r in ref])
        np.testing.assert_array_equal(d["trials"].cpu().numpy(), [r["trials"] for r in ref])
        np.testing.assert_array_equal(d["hist"].cpu().numpy(), np.stack([r["hist"] for r in ref]))
        got_lng = d["lng"].cpu().numpy()
        assert np.array_equal(got_lng, np.stack([r["lng"] for r in ref]), equal_nan=True)
        if q == 0:
            np.testing.assert_array_equal(d["order"].cpu().numpy(), [r["order"][0] for r in ref])
        else:
            np.testing.assert_array_equal(d["order"].cpu().numpy(), np.concatenate([r["order"] for r in ref]))
    # the configurations stay consistent with their levels and orders
    for w, r in enumerate(ref):
        assert lv.index(model.energy(r["s"])) == r["idx"]
        assert windows[w][0] <= r["idx"] <= windows[w][1]


@pytest.mark.parametrize("kind,shape,q", [("ising", (8, 8), 0), ("potts", (6, 5), 5)])
def test_shared_and_global_paths_agree_over_many_blocks(cuda, kind, shape, q):
    """70 walkers: three blocks of the shared-memory kernel, the last one partial."""
    model = _model(kind, shape, q)
    out = []
    for memory in ("shared", "global"):
        wl = WangLandau(model, seed=21, n_walkers=70)
        W = wl.walkers
        lng = torch.zeros((70, wl.levels.size), dtype=torch.float64, device=cuda)
        lnf = torch.full((70,), 0.01, dtype=torch.float64, device=cuda)
        one_t = torch.tensor([w % 2 for w in range(70)], dtype=torch.int32, device=cuda)
        for _ in range(3):
            W.run(0, lng, 5 * model.n_sites, ln_f=lnf, n_levels=lnf * 100, one_over_t=one_t,
                  t_base=torch.zeros(70, dtype=torch.int64, device=cuda), memory=memory)
        out.append([x.cpu().numpy() for x in (lng, W.hist, W.spins, W.idx, W.order, W.trials)])
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("kind,shape,q,win", [
    ("ising", (8, 8), 0, (-1.9, -1.6)), ("ising", (4, 4, 4), 0, (-2.0, -1.5)), ("ising", (16,), 0, (-0.9, -0.5)),
    ("potts", (8, 8), 10, (-1.95, -0.6)), ("potts", (6, 5), 4, (-1.5, -1.2)), ("potts", (4, 4, 2), 3, (-2.5, -1.5))])
def test_descent_into_window_bit_identical_to_oracle(cuda, kind, shape, q, win):
    """critmc_fh_descend against the oracle for 40 walkers, and the walkers it sets up."""
    model = _model(kind, shape, q)
    lv = EnergyLevels.of(model)
    lo, hi = lv.window(*win)
    rng = np.random.default_rng(zlib.crc32(repr((kind, shape)).encode()))
    W = 40
    states = [model.initial_state("random", rng).astype(np.int8) for _ in range(W)]
    keys = rng.integers(0, 1 << 32, size=(W, 2), dtype=np.uint64).astype(np.uint32)
    idx0 = [lv.index(model.energy(st)) for st in states]
    orders = [initial_order(st, q) for st in states]
    spins = torch.from_numpy(np.stack(states)).to(cuda)
    idx = torch.tensor(idx0, dtype=torch.int64, device=cuda)
    order = torch.from_numpy(np.concatenate(orders)).to(cuda)
    window = torch.tensor([[lo, hi]] * W, dtype=torch.int32, device=cuda)
    steps = torch.empty(W, dtype=torch.int64, device=cuda)
    dkeys = torch.from_numpy(keys.view(np.int32)).to(cuda)
    lx, ly, lz = tuple(shape) + (1,) * (3 - len(shape))
    _lib.call("critmc_fh_descend", ptr(spins), len(shape), lx, ly, lz, q, W, ptr(dkeys), lv.size, ptr(idx),
              ptr(order), ptr(window), 10**6, ptr(steps), stream_handle(cuda))
    got_s, got_i, got_o, got_n = (t.cpu().numpy() for t in (spins, idx, order, steps))
    got_o = got_o.reshape(W, -1)
    for w in range(W):
        i_ref, n_ref = oracle.fh_descend(states[w], shape, q, keys[w], idx0[w], orders[w], (lo, hi), 10**6)
        np.testing.assert_array_equal(got_s[w], states[w])
        assert got_i[w] == i_ref and got_n[w] == n_ref
        np.testing.assert_array_equal(got_o[w], orders[w])
    # the drivers start every walker inside its window (random start, else the
    # ordered one), at its configuration's level
    wl = WangLandau(model, e_window=win, seed=3, n_walkers=64)
    s_all = wl.walkers.spins.cpu().numpy()
    i_all = wl.walkers.idx.cpu().numpy()
    for w in range(0, 64, 7):
        assert lo <= i_all[w] <= hi and i_all[w] == lv.index(model.energy(s_all[w]))


def _start(walkers, w):
    return (walkers.spins[w].cpu().numpy().copy(), int(walkers.idx[w]), walkers.keys[w].cpu().numpy().view(np.uint32))


def test_wang_landau_matches_replay(cuda):
    model = Ising(square(4))
    wl = WangLandau(model, seed=1)
    s, idx, key = _start(wl.walkers, 0)
    res = wl.run(1e-4, checkpoints=[1000, 50_000, 10**9])
    lv = res.levels
    r = replay_wang_landau((4, 4), 0, s, key, idx, wl.window, lv.size, 16, 1e-4, checkpoints=[1000, 50_000, 10**9])
    np.testing.assert_array_equal(wl.state, r["state"])
    assert wl.idx == r["idx"]
    assert np.array_equal(res.ln_g, r["ln_g"])
    assert np.array_equal(res.visited, r["visited"])
    assert res.trials == r["trials"] and res.ln_f == r["ln_f"] and res.stages == r["stages"]
    assert [c[0] for c in res.checkpoints] == [1000, 50_000, 10**9]
    for a, b in zip(res.checkpoints, r["checkpoints"]):
        assert a[1] == b[1] and np.array_equal(a[2], b[2])


def test_wang_landau_batch_of_windows_matches_replay(cuda):
    model = Potts(square(4, 3), 3)
    wins = [None, (-2.0, -1.0), (-1.5, -0.5), (None, -0.8)]
    wl = WangLandau(model, e_window=wins, n_walkers=4, seed=2, criterion="visit")
    starts = [_start(wl.walkers, w) for w in range(4)]
    results = wl.run(1e-3, one_over_t=True, check_sweeps=50)
    assert len(results) == 4
    for w, res in enumerate(results):
        s, idx, key = starts[w]
        r = replay_wang_landau((4, 3), 3, s, key, idx, wl.windows[w], res.levels.size, 12, 1e-3, check_sweeps=50,
                               criterion="visit")
        assert res.window == wl.windows[w]
        assert np.array_equal(res.ln_g, r["ln_g"]), w
        assert res.trials == r["trials"] and res.stages == r["stages"]
    # walkers that finished first were frozen during the run; their windows are back
    np.testing.assert_array_equal(wl.walkers.window.cpu().numpy(), np.array(wl.windows))
    assert wl.state.shape == (4, 12) and len(wl.idx) == 4


@pytest.mark.parametrize("n_walkers", [1, 4])
def test_multicanonical_matches_replay(cuda, n_walkers):
    model = Ising(square(6))
    lng = ising_log_g_square6()
    mu = Multicanonical(model, lng, seed=8, n_walkers=n_walkers)
    starts = [_start(mu.walkers, w) for w in range(n_walkers)]
    out = mu.run(3000, sweeps_per_meas=2, n_therm=50)
    outs = out if n_walkers > 1 else [out]
    for w, o in enumerate(outs):
        s, idx, key = starts[w]
        r = replay_multicanonical((6, 6), 0, s, key, idx, mu.window, mu.ln_w, 72, 3000, n_therm=50)
        np.testing.assert_array_equal(o.level_series, r["level_series"])
        np.testing.assert_array_equal(o.order_series, r["order_series"])
        np.testing.assert_array_equal(o.hist, r["hist"])


# ---- critmc's statistical checks (tests/test_flathist.py): the same cases,
# seeds and bounds, written for this package ----

EXACT_6 = None


def _exact_6():
    global EXACT_6
    if EXACT_6 is None:
        EXACT_6 = ising_log_g_square6()
    return EXACT_6


@pytest.mark.parametrize("one_over_t", [False, True])
def test_wang_landau_ising_against_exact_dos(cuda, one_over_t):
    """6x6 Ising to ln f = 1e-6: levels seen = levels that exist; mean |ln g error|
    below 0.02 (1/t) or 0.08 (plain, which saturates); canonical energies within
    0.01 / 0.03 of Kaufman's at beta 0.3, 0.44, 0.6."""
    result = WangLandau(Ising(square(6)), seed=3, criterion="flat").run(1e-6, one_over_t=one_over_t)
    reference = _exact_6()
    seen = result.visited
    assert (seen == np.isfinite(reference)).all()
    deviation = np.abs(result.normalized()[seen] - reference[seen]).mean()
    assert deviation < {True: 0.02, False: 0.08}[one_over_t]
    betas = (0.3, 0.44, 0.6)
    kaufman = np.array([kaufman_energy(b, 6) for b in betas])
    bound = {True: 0.01, False: 0.03}[one_over_t] + 1e-5 * np.abs(kaufman)  # numpy allclose's test
    assert (np.abs(result.canonical(list(betas))["u"] - kaufman) <= bound).all()


def test_wang_landau_batch_of_seeds_against_exact_dos(cuda):
    """Independent walkers in one launch: each converges, and their spread is the error bar."""
    results = WangLandau(Ising(square(6)), seed=11, n_walkers=64).run(1e-5)
    reference = _exact_6()
    on = np.isfinite(reference)
    per_walker = np.array([np.abs(r.normalized()[on] - reference[on]).mean() for r in results])
    assert per_walker.max() < 0.08 and np.median(per_walker) < 0.04
    pooled = np.mean([r.normalized()[on] for r in results], axis=0)
    assert np.abs(pooled - reference[on]).mean() < 0.01


def test_wang_landau_checkpoints_and_stages(cuda):
    marks = [10_000, 100_000, 1_000_000]
    result = WangLandau(Ising(square(4)), seed=1).run(1e-5, checkpoints=marks)
    assert [trials for trials, _, _ in result.checkpoints] == marks
    assert len(result.stages) > 0 and result.stages[0]["ln_f"] == 1.0


def test_wang_landau_potts_window(cuda):
    """4x3 q=3 Potts in the window [-2, -1] per site: ln g differences as the exact
    joint DOS (spread below 0.02), no level above E = -12."""
    joint = JointDOS("potts3_dos_square4x3")
    exact = {float(e): float(np.log(c)) for e, c in zip(joint.energies, joint.counts.sum(axis=1))}
    result = WangLandau(Potts(square(4, 3), 3), e_window=(-2.0, -1.0), seed=4).run(1e-7)
    energies = result.levels.energies[result.visited]
    offsets = result.normalized()[result.visited] - np.array([exact[float(e)] for e in energies])
    assert offsets.max() - offsets.min() < 0.02
    assert energies.max() <= -12


def test_multicanonical_reweighting_to_canonical(cuda):
    """Exact 1/g weights on 6x6 Ising: every level is sampled and the reweighted energy
    is Kaufman's within 0.01 at beta 0.3, 0.44, 0.55."""
    reference = _exact_6()
    series = Multicanonical(Ising(square(6)), reference, seed=8).run(200_000, sweeps_per_meas=1, n_therm=100)
    assert np.count_nonzero(series.hist) == np.count_nonzero(np.isfinite(reference))
    for beta in (0.3, 0.44, 0.55):
        assert abs(series.canonical(beta)["u"][0] - kaufman_energy(beta, 6)) <= 0.01


# Equal-height point of the q = 10 Potts 8 x 8 torus in the window [-1.95, -0.6]
# (split -1.3): critmc's own Wang-Landau converged to ln f = 1e-6, four seeds
# (fixture).  It lies 0.047 below beta_c, so critmc's own test bracket
# beta_c +- 0.05 (tests/test_flathist.py:69-81) holds the root only 0.003 from
# its edge; the bracket here is wider and the root is checked against it.


def test_multicanonical_potts_double_peak(cuda):
    from exact_helpers import golden

    model = Potts(square(8), 10)
    window = (-1.95, -0.6)
    estimate = WangLandau(model, e_window=window, seed=9).run(1e-5)
    series = Multicanonical(model, estimate.ln_g, e_window=window, seed=10).run(100_000)
    beta_c = float(golden()["potts_beta_c"]["10"])
    beta = series.equal_height_beta((beta_c - 0.1, beta_c + 0.05), split=-1.3)
    peaks = series.double_peak(beta, split=-1.3)
    assert abs(peaks["p_ordered"] / peaks["p_disordered"] - 1.0) < 1e-6
    assert peaks["e_ordered"] < -1.5 and peaks["e_disordered"] > -1.1
    assert abs(beta - golden()["potts10_L8_equal_height"]["beta"]) < 0.015
    assert abs(beta - beta_c) < 0.065


def _estimate_with_level_12_unvisited():
    """A converged 6x6 Ising estimate altered so that level 12 looks never reached:
    ln g there is 0, Wang-Landau's starting value."""
    estimate = WangLandau(Ising(square(6)), seed=3).run(1e-5)
    assert estimate.visited[12]
    estimate.ln_g[12] = 0.0
    estimate.visited[12] = False
    return estimate


def test_multicanonical_raw_ln_g_traps_the_walk_on_an_unvisited_level(cuda):
    """Given the bare array, the unvisited level's weight 1/g = 1 dwarfs all others."""
    estimate = _estimate_with_level_12_unvisited()
    series = Multicanonical(Ising(square(6)), estimate.ln_g, seed=4).run(5000)
    assert series.hist[12] / series.hist.sum() > 0.99


def test_multicanonical_forbids_levels_wang_landau_never_visited(cuda):
    """Given the result object, the unvisited level is forbidden and the others are
    sampled about equally (none below 30 % of the mean)."""
    estimate = _estimate_with_level_12_unvisited()
    series = Multicanonical(Ising(square(6)), estimate, seed=4).run(50_000)
    assert series.hist[12] == 0
    sampled = series.hist > 0
    assert (sampled == estimate.visited).all()
    counts = series.hist[sampled]
    assert counts.min() > 0.3 * counts.mean()


def test_multicanonical_wl_result_matches_its_array_when_all_levels_were_visited(cuda):
    model = Potts(square(6), 10)
    window = (-1.95, -0.6)
    estimate = WangLandau(model, e_window=window, seed=9).run(1e-4)
    from_array = Multicanonical(model, estimate.ln_g, e_window=window, seed=10).run(5000)
    from_result = Multicanonical(model, estimate, e_window=window, seed=10).run(5000)
    np.testing.assert_array_equal(from_array.level_series, from_result.level_series)
