"""Work items advanced by teams: a thread-block cluster of 2, 4, 8 or 16 blocks
per item (the lattice in global memory, the cluster barrier between colours)
gives, bit for bit, what one block per item and the per-model entry points
give, for every model family, alone or mixed with items of other team sizes,
and stops under a control like one block does."""

from __future__ import annotations

import time

import numpy as np
import pytest
import torch

from critmc_b200 import ON, Ising, Potts, hypercubic, square
from critmc_b200.control import CANCELLED, TIMEOUT, RunControl
from critmc_b200.items import ITEM_BYTE_ISING, ITEM_MSC_ISING, ITEM_ON, ITEM_POTTS, ItemRun, run_items, team_clusters

from test_gpu_items import MIX, _assert_same, _pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("team", [2, 4, 8, 16])
def test_team_items_match_per_model_runs(cuda, team):
    pairs = [_pair(i, f, s, cuda) for i, (f, s, _, _) in enumerate(MIX)]
    buf = None
    for n_meas in (4, 3):  # two slices: the sweep counters carry over
        alone = [m.advance(c[0], r[0], beta, np.array(sched), n_meas)
                 for (m, c, r), (_, _, sched, beta) in zip(pairs, MIX)]
        items = [ItemRun(m, c[1], r[1], beta, np.array(sched), n_meas, team=team)
                 for (m, c, r), (_, _, sched, beta) in zip(pairs, MIX)]
        buf = run_items(items, cuda, buffer=buf)
        mixed = [it.finish() for it in items]
        for (model, chains, runs), a, b in zip(pairs, alone, mixed):
            _assert_same(a, b)
            _assert_same({k: np.asarray(v) for k, v in runs[0].items()},
                         {k: np.asarray(v) for k, v in runs[1].items()})
    for model, chains, _ in pairs:
        np.testing.assert_array_equal(chains[0].fetch(), chains[1].fetch())


def test_mixed_team_sizes_in_one_call(cuda):
    """Each item its own team size: one launch group per (family, team)."""
    sizes = [1, 2, 4, 8, 16]
    pairs = [_pair(i, f, s, cuda) for i, (f, s, _, _) in enumerate(MIX)]
    alone = [m.advance(c[0], r[0], beta, np.array(sched), 6)
             for (m, c, r), (_, _, sched, beta) in zip(pairs, MIX)]
    items = [ItemRun(m, c[1], r[1], beta, np.array(sched), 6, team=sizes[i % len(sizes)])
             for i, ((m, c, r), (_, _, sched, beta)) in enumerate(zip(pairs, MIX))]
    run_items(items, cuda)
    for (model, chains, _), a, it in zip(pairs, alone, items):
        _assert_same(a, it.finish())
        np.testing.assert_array_equal(chains[0].fetch(), chains[1].fetch())


@pytest.mark.parametrize("shape,team", [((2048, 2048), 16), ((256, 128, 64), 8)])
def test_team_msc_items_above_the_one_block_limit(cuda, shape, team):
    """Teams keep multi-spin-coded lattices in global memory, so they take
    lattices above the 2^20 sites one block holds in shared memory."""
    model = Ising(hypercubic(shape))
    s0 = model.initial_state("random", np.random.default_rng(3))
    a = model.to_device(s0, np.random.default_rng(9), cuda)
    b = model.to_device(s0, np.random.default_rng(9), cuda)
    ra, rb = model.begin(s0), model.begin(s0)
    beta = 0.4406868 if len(shape) == 2 else 0.2216546
    for sched in ([[0, 1]], [[2, 2]]):
        x = model.advance(a, ra, beta, np.array(sched), 3)
        it = ItemRun(model, b, rb, beta, np.array(sched), 3, team=team)
        run_items([it], cuda)
        _assert_same(x, it.finish())
    np.testing.assert_array_equal(a.fetch(), b.fetch())


def test_potts_and_on_teams_long_slices(cuda):
    """Many measurements per item: the per-measurement sums of the blocks and
    the Potts count snapshots alternate between two buffers."""
    cases = [(Potts(square(128), 10), 1.42, [[0, 1]], 8), (Potts(square(96, 64), 3), 1.0, [[2, 1]], 4),
             (ON(square(128), 2), 1.1, [[0, 1]], 16), (ON(square(64), 3), 0.7, [[2, 1], [5, 4]], 8)]
    for k, (model, beta, sched, team) in enumerate(cases):
        s0 = model.initial_state("random", np.random.default_rng(20 + k))
        a = model.to_device(s0, np.random.default_rng(40 + k), cuda)
        b = model.to_device(s0, np.random.default_rng(40 + k), cuda)
        ra, rb = model.begin(s0), model.begin(s0)
        x = model.advance(a, ra, beta, np.array(sched), 57)
        it = ItemRun(model, b, rb, beta, np.array(sched), 57, team=team)
        run_items([it], cuda)
        _assert_same(x, it.finish())
        _assert_same({q: np.asarray(v) for q, v in ra.items()}, {q: np.asarray(v) for q, v in rb.items()})
        np.testing.assert_array_equal(a.fetch(), b.fetch())


def test_team_items_stop_on_budget_and_on_cancel(cuda):
    model = Ising(square(1024, 256))
    rng = np.random.default_rng(4)

    def items():
        out = []
        for i in range(24):
            s0 = model.initial_state("random", rng)
            ch = model.to_device(s0, np.random.default_rng(100 + i), cuda)
            out.append(ItemRun(model, ch, model.begin(s0), 0.44, np.array([[0, 20]]), 10000, team=8))
        return out

    ctl = RunControl(cuda).arm(2e-3)
    runs = items()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run_items(runs, cuda, control=ctl)
    e1.record()
    assert ctl.wait() == TIMEOUT
    assert e0.elapsed_time(e1) * 1e-3 < 0.15
    runs = items()
    ctl.arm(None)
    e0.record()
    run_items(runs, cuda, control=ctl)
    e1.record()
    time.sleep(0.05)
    ctl.cancel()
    assert ctl.wait() == CANCELLED
    assert e0.elapsed_time(e1) * 1e-3 < 0.2
    # the device is still usable and teams still give the per-model results
    pairs = [_pair(i, f, s, cuda) for i, (f, s, _, _) in enumerate(MIX[:4])]
    alone = [m.advance(c[0], r[0], beta, np.array(sched), 2)
             for (m, c, r), (_, _, sched, beta) in zip(pairs, MIX[:4])]
    its = [ItemRun(m, c[1], r[1], beta, np.array(sched), 2, team=4)
           for (m, c, r), (_, _, sched, beta) in zip(pairs, MIX[:4])]
    run_items(its, cuda)
    for a, it in zip(alone, its):
        _assert_same(a, it.finish())


def test_team_capacity_query(cuda):
    """The server asks which team sizes the GPU schedules: on a B200 every
    family runs clusters of up to 16 blocks, several at once."""
    for kind, n, dim in ((ITEM_MSC_ISING, 0, 2), (ITEM_BYTE_ISING, 0, 2), (ITEM_POTTS, 10, 2), (ITEM_ON, 2, 2),
                         (ITEM_ON, 3, 3)):
        counts = [team_clusters(kind, n, dim, t, cuda) for t in (2, 4, 8, 16)]
        assert all(c >= 1 for c in counts), (kind, n, dim, counts)
        assert counts == sorted(counts, reverse=True)
