"""Library-held chains (handle ABI) and the batch queue: the same series as the
per-model entry points for the same key, state and sweep counter."""

from __future__ import annotations

import numpy as np
import pytest

from critmc_b200 import ON, Ising, Potts, hypercubic
from critmc_b200.byte_models import IsingByteChain, PottsChain
from critmc_b200.chains import Batch, Chain
from critmc_b200.models import _IsingMscChain
from critmc_b200.on_models import ONChain

pytestmark = pytest.mark.gpu

CASES = [
    ("ising", (128, 64), 0, 0.0, "metropolis", 0.44),
    ("ising", (64, 16, 8), 0, 0.2, "heatbath+metropolis", 0.22),
    ("ising", (18, 10), 0, 0.0, "metropolis", 0.44),
    ("ising", (64,), 0, 0.0, "heatbath", 0.7),
    ("potts", (16, 16), 5, 0.0, "metropolis+heatbath", 1.1),
    ("on", (16, 16), 2, 0.0, "heatbath+2*overrelax", 1.1),
    ("on", (8, 8, 8), 3, 0.0, "metropolis", 0.7),
]


def _reference(kind, shape, q_or_n, h, state, key, cuda):
    lat = hypercubic(shape)
    if kind == "ising":
        model = Ising(lat, h)
        msc = len(shape) >= 2 and shape[0] % 64 == 0
        chain = (_IsingMscChain if msc else IsingByteChain)(model, state, key, cuda)
    elif kind == "potts":
        model = Potts(lat, q_or_n)
        chain = PottsChain(model, state, key, cuda)
    else:
        model = ON(lat, q_or_n)
        chain = ONChain(model, state, key, cuda, lane="block")
    return model, chain, model.begin(state)


@pytest.mark.parametrize("kind,shape,q_or_n,h,updates,beta", CASES)
def test_chain_handle_equals_per_model_entry_points(cuda, kind, shape, q_or_n, h, updates, beta):
    ch = Chain(kind, shape, q_or_n=q_or_n, h=h, seed=12345, chain_id=7, device=cuda)
    s0, run0 = ch.state()
    info = ch.info()
    model, ref, running = _reference(kind, shape, q_or_n, h, s0, info["key"], cuda)
    if run0 is not None:
        assert run0[0] == running["e_b" if kind == "ising" else "energy"]
    from critmc_b200.chains import schedule_array

    sched = schedule_array(updates)
    for n in (4, 3):
        got = ch.advance(beta, updates, n)
        want = model.advance(ref, running, beta, sched, n)
        for k, v in got.items():
            np.testing.assert_array_equal(v, want[k], err_msg=k)
    s1, run1 = ch.state()
    np.testing.assert_array_equal(s1, ref.fetch().astype(s1.dtype))
    assert ch.info()["sweep"] == ref.sweep
    if kind == "ising":
        assert (run1[0], run1[1]) == (running["e_b"], running["m"])
    ch.close()


def test_random_start_is_keyed_and_set_state_round_trips(cuda):
    a = Chain("potts", (16, 8), q_or_n=4, seed=1, chain_id=0, device=cuda)
    b = Chain("potts", (16, 8), q_or_n=4, seed=1, chain_id=0, device=cuda)
    c = Chain("potts", (16, 8), q_or_n=4, seed=1, chain_id=1, device=cuda)
    np.testing.assert_array_equal(a.state()[0], b.state()[0])
    assert not np.array_equal(a.state()[0], c.state()[0])
    s = np.random.default_rng(0).integers(0, 4, 128).astype(np.int8)
    a.set_state(s)
    got, run = a.state()
    np.testing.assert_array_equal(got, s)
    ref = Potts(hypercubic((16, 8)), 4).begin(s)
    assert run[0] == ref["energy"]
    np.testing.assert_array_equal(run[1:], ref["counts"])
    o = Chain("ising", (256, 256), device=cuda, start="ordered")
    st, run = o.state()
    assert (st == 1).all() and run[0] == -2 * 256 * 256 and run[1] == 256 * 256
    with pytest.raises(Exception):
        a.set_state(np.full(128, 9, dtype=np.int8))


def test_batch_queue_equals_sequential_advances(cuda):
    specs = [("ising", (64, 64), 0), ("ising", (1024, 1024), 0), ("potts", (32, 32), 10),
             ("on", (32, 32), 2), ("ising", (20, 20), 0)]
    mk = lambda: [Chain(k, s, q_or_n=q, seed=99, chain_id=i, device=cuda) for i, (k, s, q) in enumerate(specs)]
    seq, bat = mk(), mk()
    batch = Batch(cuda)
    tickets = []
    for rnd in range(2):  # two submissions per chain: they run in order
        for i, ch in enumerate(bat):
            tickets.append((rnd, i, batch.submit(ch, 0.44 if specs[i][0] != "potts" else 1.4, "metropolis", 5 + rnd)))
    extra = batch.submit(bat[0], 0.44, "metropolis", 3)
    batch.cancel(extra)
    assert batch.pending() == 2 * len(specs)
    res = batch.poll()
    assert batch.pending() == 0 and len(res) == 2 * len(specs)
    for rnd, i, t in tickets:
        want = seq[i].advance(0.44 if specs[i][0] != "potts" else 1.4, "metropolis", 5 + rnd)
        for k, v in want.items():
            np.testing.assert_array_equal(res[t][k], v, err_msg=f"{specs[i]} {k}")
    for a, b in zip(seq, bat):
        np.testing.assert_array_equal(a.state()[0], b.state()[0])
