"""O(n) kernels: agreement with the FP32 CPU replay, and critmc's exact ring results."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import assert_consistent
from exact_helpers import golden

import oracle
from critmc_b200 import ON, Simulation, chain, hypercubic, square
from critmc_b200.on_models import ONChain

pytestmark = pytest.mark.gpu

# Spins are bit-identical (shared elementary functions, no contraction) and the
# observables are exact fixed-point sums on both sides, so everything agrees
# bit for bit (the bar for FP32 O(n) is 1e-5 relative).

CASES = [
    ((16, 16), 2, [[2, 1], [5, 4]], 1.0),
    ((16, 16), 2, [[0, 1]], 1.1),
    ((16, 16), 3, [[2, 1], [5, 4]], 0.7),
    ((16, 16), 3, [[0, 2]], 0.9),
    ((8, 6, 4), 3, [[2, 1], [5, 1]], 0.7),
    ((32,), 2, [[2, 1], [0, 1], [5, 2]], 1.1),
    ((128, 130), 2, [[2, 1]], 1.0),  # larger than shared memory: updated in HBM
    ((64, 64), 3, [[0, 1]], 0.9),  # 48 KiB lattice: with the block's static arrays above the default limit
]


@pytest.mark.parametrize("lane", ["block", "grid"])
@pytest.mark.parametrize("shape,n,sched,beta", CASES)
def test_on_agrees_with_replay(cuda, shape, n, sched, beta, lane):
    model = ON(hypercubic(shape), n)
    rng = np.random.default_rng(n * 7 + len(shape))
    s0 = model.initial_state("random", rng).astype(np.float32)
    key = rng.integers(0, 2**32, 2, dtype=np.uint64).astype(np.uint32)
    ch = ONChain(model, s0, key, cuda, lane=lane)
    running = {"step": 0.8}
    parts = [ch.advance(running, beta, np.array(sched), k) for k in (13, 7)]
    raw = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    s_ref = s0.copy()
    e, m, sc, ss, aux = oracle.on_run(s_ref, shape, n, key, beta, 0.8, sched, 20)
    np.testing.assert_array_equal(raw["E"], e)
    np.testing.assert_array_equal(raw["M"], m)
    np.testing.assert_array_equal(raw["stiff_c"], sc)
    np.testing.assert_array_equal(raw["stiff_s"], ss)
    np.testing.assert_array_equal(ch.fetch().astype(np.float32), s_ref)
    np.testing.assert_array_equal(raw["aux"], aux)


@pytest.mark.parametrize("blocks", [1, 3, 0])
def test_on_grid_lane_any_block_count(cuda, blocks):
    """The multi-block lane gives the block lane's results for any split, long runs included."""
    model = ON(hypercubic((64, 64)), 2)
    rng = np.random.default_rng(11)
    s0 = model.initial_state("random", rng).astype(np.float32)
    key = np.array([5, 6], dtype=np.uint32)
    a = ONChain(model, s0, key, cuda, lane="block")
    b = ONChain(model, s0, key, cuda, lane="grid")
    b.blocks_per_chain = blocks
    sched = np.array([[2, 1], [5, 2]])
    ra = a.advance({"step": 1.0}, 1.1, sched, 300)  # > one graph of measurements
    rb = b.advance({"step": 1.0}, 1.1, sched, 300)
    for k in ra:
        np.testing.assert_array_equal(ra[k], rb[k], err_msg=k)
    np.testing.assert_array_equal(a.fetch(), b.fetch())


@pytest.mark.parametrize("n_comp", [2, 3])
@pytest.mark.parametrize("updates", ["metropolis", "heatbath", "metropolis+3*overrelax"])
def test_on_ring_matches_transfer_operator(cuda, n_comp, updates):
    """critmc tests/test_kernels.py:95-109."""
    ref = golden()["on_ring"][f"n{n_comp}_N8_b1.1"]
    beta, n_sites = 1.1, 8
    sim = Simulation(ON(chain(n_sites), n_comp), beta, updates, seed=5)
    sim.thermalize(2000)
    ts = sim.run(100_000)
    assert_consistent(ts["e"], ref["energy"])
    e = ts["E"]
    assert beta ** 2 * e.var() / n_sites == pytest.approx(ref["specific_heat"], rel=0.06)


def test_on_state_stays_normalised_and_energy_consistent(cuda):
    """critmc tests/test_kernels.py:112-118 (without the cluster moves)."""
    lat = square(6)
    sim = Simulation(ON(lat, 3), 0.7, "metropolis+2*overrelax+heatbath", seed=1)
    sim.thermalize(200)
    ts = sim.run(200)
    s = sim.state
    assert np.allclose(np.linalg.norm(s, axis=1), 1.0, atol=1e-6)
    assert ts["E"][-1] == pytest.approx(ON(lat, 3).energy(s), rel=1e-6)


def test_metropolis_step_is_tuned(cuda):
    sim = Simulation(ON(square(8), 2), 1.0, "metropolis", seed=2)
    info = sim.thermalize(500)
    assert 0.001 <= info["step"] <= 10
    acc = sim.run(500).meta["acceptance"]
    assert 0.3 < acc < 0.7


def test_on_ensemble_chain_equals_single_chain(cuda):
    """A chain of the batched ensemble gives the series of the same chain run alone."""
    from critmc_b200.on_models import ONEnsemble
    from critmc_b200.rng import make_rng, philox_key

    model = ON(hypercubic((32, 32)), 2)
    temps = np.linspace(0.7, 1.1, 4)
    ens = ONEnsemble(model, temps, 3, seed=9, device=cuda)
    sched = np.array([[2, 1], [5, 4]])
    out = ens.run(6, sched)
    for t, c in ((0, 0), (2, 1), (3, 2)):
        rng = make_rng(9, "on", 2, 32, t, c)
        s0 = model.initial_state("random", rng).astype(np.float32)
        ch = ONChain(model, s0, philox_key(rng), cuda, lane="block")
        raw = ch.advance({"step": 1.0}, 1.0 / temps[t], sched, 6)
        i = t * 3 + c
        np.testing.assert_array_equal(out["E"][i].cpu().numpy(), raw["E"])
        np.testing.assert_array_equal(out["M"][i].cpu().numpy(), raw["M"])
        np.testing.assert_array_equal(ens.chain(i), ch.fetch())
