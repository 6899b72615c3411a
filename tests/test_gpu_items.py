"""Work items: chains of every model family and many sizes advanced by one
``critmc_run_items`` call give, bit for bit, what the per-model entry points
give for each chain alone."""

from __future__ import annotations

import numpy as np
import pytest

from critmc_b200 import ON, Ising, Potts, hypercubic
from critmc_b200.items import ItemRun, run_items

pytestmark = pytest.mark.gpu

# (model factory, shape, schedule, beta)
MIX = [
    (lambda l: Ising(l), (128, 64), [[0, 1]], 0.4406868),
    (lambda l: Ising(l, 0.3), (64, 32), [[2, 1]], 0.35),
    (lambda l: Ising(l), (64, 16, 8), [[0, 2], [2, 1]], 0.2216546),
    (lambda l: Ising(l, -0.1), (256, 256), [[0, 1]], 0.5),
    (lambda l: Ising(l), (18, 10), [[0, 1]], 0.44),
    (lambda l: Ising(l, 0.25), (6, 4, 8), [[2, 1]], 0.2),
    (lambda l: Ising(l), (64,), [[2, 1]], 0.7),
    (lambda l: Ising(l), (640, 322), [[0, 1]], 0.44),  # byte lattice above the shared-memory limit
    (lambda l: Potts(l, 3), (32, 32), [[2, 1]], 1.0),
    (lambda l: Potts(l, 10), (8, 8, 8), [[0, 1]], 0.6),
    (lambda l: Potts(l, 4), (64,), [[2, 2]], 0.8),
    (lambda l: Potts(l, 10), (400, 300), [[2, 1], [0, 1]], 1.42),
    (lambda l: ON(l, 2), (16, 16), [[0, 1], [5, 2]], 1.1),
    (lambda l: ON(l, 3), (8, 8, 8), [[2, 1], [5, 1]], 0.69),
    (lambda l: ON(l, 2), (32,), [[2, 1]], 2.0),
    (lambda l: ON(l, 3), (96, 96), [[0, 1]], 0.7),
]


def _pair(i, factory, shape, cuda):
    """Two chains with the same lattice, key and running sums."""
    model = factory(hypercubic(shape))
    rng = np.random.default_rng(1000 + i)
    s0 = model.initial_state("random", rng)
    chains = [model.to_device(s0, np.random.default_rng(77 + i), cuda) for _ in range(2)]
    return model, chains, [model.begin(s0), model.begin(s0)]


def _assert_same(a: dict, b: dict):
    assert set(a) == set(b)
    for k in a:
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)


@pytest.mark.parametrize("smem_limit", [0, 16 * 1024])
def test_mixed_items_match_per_model_runs(cuda, smem_limit):
    pairs = [_pair(i, f, s, cuda) for i, (f, s, _, _) in enumerate(MIX)]
    buf = None
    for n_meas in (5, 3):  # two slices: the sweep counters carry over
        alone = [m.advance(c[0], r[0], beta, np.array(sched), n_meas)
                 for (m, c, r), (_, _, sched, beta) in zip(pairs, MIX)]
        items = [ItemRun(m, c[1], r[1], beta, np.array(sched), n_meas)
                 for (m, c, r), (_, _, sched, beta) in zip(pairs, MIX)]
        buf = run_items(items, cuda, smem_limit=smem_limit, buffer=buf)
        mixed = [it.finish() for it in items]
        for (model, chains, runs), a, b in zip(pairs, alone, mixed):
            _assert_same(a, b)
            assert chains[0].sweep == chains[1].sweep
            _assert_same({k: np.asarray(v) for k, v in runs[0].items()},
                         {k: np.asarray(v) for k, v in runs[1].items()})
    for model, chains, _ in pairs:
        np.testing.assert_array_equal(chains[0].fetch(), chains[1].fetch())


def test_items_order_does_not_matter(cuda):
    """A chain gives the same series whatever it is batched with, in any order."""
    sel = [0, 4, 8, 12, 9, 13, 2]
    pairs = [_pair(i, MIX[i][0], MIX[i][1], cuda) for i in sel]
    out = []
    for copy, order in ((0, sel), (1, sel[::-1])):
        idx = {i: k for k, i in enumerate(sel)}
        items = {i: ItemRun(pairs[idx[i]][0], pairs[idx[i]][1][copy], pairs[idx[i]][2][copy],
                            MIX[i][3], np.array(MIX[i][2]), 4) for i in order}
        run_items([items[i] for i in order], cuda)
        out.append({i: items[i].finish() for i in order})
    for i in sel:
        _assert_same(out[0][i], out[1][i])


def test_msc_item_matches_msc_entry_point_many_chains(cuda):
    """Thousands of small MSC chains in one call (more items than resident blocks)."""
    model = Ising(hypercubic((64, 64)))
    n = 600
    rng = np.random.default_rng(5)
    states = [model.initial_state("random", rng) for _ in range(n)]
    a = [model.to_device(s, np.random.default_rng(i), cuda) for i, s in enumerate(states)]
    b = [model.to_device(s, np.random.default_rng(i), cuda) for i, s in enumerate(states)]
    ra = [model.begin(s) for s in states]
    rb = [model.begin(s) for s in states]
    alone = [model.advance(c, r, 0.4406868, np.array([[0, 1]]), 3) for c, r in zip(a[:40], ra[:40])]
    items = [ItemRun(model, c, r, 0.4406868, np.array([[0, 1]]), 3) for c, r in zip(b, rb)]
    run_items(items, cuda)
    mixed = [it.finish() for it in items]
    for x, y in zip(alone, mixed[:40]):
        _assert_same(x, y)
    for c0, c1 in zip(a[:40], b[:40]):
        np.testing.assert_array_equal(c0.fetch(), c1.fetch())
