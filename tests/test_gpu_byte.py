"""Byte-lattice kernels (int8 Ising, Potts) against the CPU replay, and the
Simulation API against critmc's exact results on the GPU."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import assert_consistent
from exact_helpers import JointDOS, kaufman_energy

import oracle
from critmc_b200 import Ising, Potts, Simulation, chain, hypercubic, square
from critmc_b200.byte_models import IsingByteChain, PottsChain

pytestmark = pytest.mark.gpu

ISING_CASES = [
    ((32, 32), [[0, 1]], 0.4406868, 0.0),
    ((32, 32), [[2, 1]], 0.4406868, 0.0),
    ((16, 6), [[0, 2], [2, 1]], 0.3, 0.25),
    ((64,), [[0, 1]], 0.7, 0.0),
    ((6, 4, 8), [[2, 1]], 0.2216546, 0.1),
    ((2, 2), [[0, 1]], 1.5, 0.0),
    ((128, 130), [[0, 1]], 0.44, 0.0),  # > shared memory: updated in HBM
]


@pytest.mark.parametrize("shape,sched,beta,h", ISING_CASES)
def test_ising_byte_bit_identical_to_replay(cuda, shape, sched, beta, h):
    model = Ising(hypercubic(shape), h)
    rng = np.random.default_rng(sum(shape))
    s0 = model.initial_state("random", rng)
    key = rng.integers(0, 2**32, 2, dtype=np.uint64).astype(np.uint32)
    chain_ = IsingByteChain(model, s0, key, cuda)
    running = model.begin(s0)
    parts = [chain_.advance(running, beta, np.array(sched), k) for k in (7, 12)]
    raw = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    s_ref = s0.copy()
    e, m, aux, run = oracle.ising_byte_run(s_ref, shape, key, beta, h, sched, 19)
    np.testing.assert_array_equal(chain_.fetch(), s_ref)
    np.testing.assert_array_equal(raw["Eb"], e)
    np.testing.assert_array_equal(raw["M"], m)
    np.testing.assert_array_equal(raw["aux"], aux)
    assert (running["e_b"], running["m"]) == (run[0], run[1])


POTTS_CASES = [
    ((32, 32), 3, [[0, 1]], 1.0),
    ((32, 32), 10, [[0, 1]], 1.42),
    ((16, 16), 10, [[2, 1]], 1.42),
    ((8, 6, 4), 4, [[2, 1], [0, 1]], 0.6),
    ((64,), 2, [[2, 2]], 0.8),
    ((16, 16), 127, [[0, 1], [2, 1]], 2.0),
]


@pytest.mark.parametrize("shape,q,sched,beta", POTTS_CASES)
def test_potts_bit_identical_to_replay(cuda, shape, q, sched, beta):
    model = Potts(hypercubic(shape), q)
    rng = np.random.default_rng(q + sum(shape))
    s0 = model.initial_state("random", rng)
    key = rng.integers(0, 2**32, 2, dtype=np.uint64).astype(np.uint32)
    ch = PottsChain(model, s0, key, cuda)
    running = model.begin(s0)
    parts = [ch.advance(running, beta, np.array(sched), k) for k in (5, 9)]
    raw = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    s_ref = s0.copy()
    e, co, aux, en, cnt = oracle.potts_run(s_ref, shape, q, key, beta, sched, 14)
    np.testing.assert_array_equal(ch.fetch(), s_ref)
    np.testing.assert_array_equal(raw["E"], e)
    np.testing.assert_array_equal(raw["counts"], co)
    np.testing.assert_array_equal(raw["aux"], aux)
    assert running["energy"] == en
    np.testing.assert_array_equal(running["counts"], cnt)


def _agrees_with_enumeration(dos, beta, series, observables, h=0.0):
    """Each named stream of ``series`` against the exact canonical average of its function."""
    for name, fn in observables.items():
        assert_consistent(series[name], dos.average(beta, fn, h=h))


@pytest.mark.parametrize("updates", ["metropolis", "heatbath"])
def test_ising_4x4_matches_enumeration(cuda, updates):
    """critmc tests/test_kernels.py:27-40, on a bipartite 4x4 torus: E, m^2 and m^4."""
    dos = JointDOS("ising_dos_square4")
    beta, sites = 0.35, 16
    sim = Simulation(Ising(square(4)), beta, updates, seed=12)
    sim.thermalize(2000)
    series = sim.run(200_000)
    _agrees_with_enumeration(dos, beta, series, {"E": lambda e, mag: e,
                                                 "m2": lambda e, mag: np.square(mag / sites),
                                                 "m4": lambda e, mag: np.power(mag / sites, 4)})
    final = sim.state
    assert sim.running["e_b"] == Ising(square(4)).bond_energy(final)
    assert sim.running["m"] == int(np.sum(final, dtype=np.int64))


@pytest.mark.parametrize("updates", ["metropolis", "heatbath"])
def test_ising_in_a_field(cuda, updates):
    """critmc tests/test_kernels.py:55-70: E and m at h = 0.4."""
    dos = JointDOS("ising_dos_square4")
    beta, field = 0.3, 0.4
    sim = Simulation(Ising(square(4), h=field), beta, updates, seed=8)
    sim.thermalize(1000)
    series = sim.run(150_000)
    _agrees_with_enumeration(dos, beta, series, {"E": lambda e, mag: e - field * mag,
                                                 "m": lambda e, mag: mag / 16}, h=field)


@pytest.mark.parametrize("updates", ["metropolis", "heatbath"])
def test_potts_matches_enumeration(cuda, updates):
    """critmc tests/test_kernels.py:78-92, on a bipartite 4x2 torus: E and m^2 (the
    fixture's order variable is q sum_k n_k^2)."""
    dos = JointDOS("potts3_dos_square4x2")
    beta, q, sites = 0.8, 3, 8
    sim = Simulation(Potts(square(4, 2), q), beta, updates, seed=21)
    sim.thermalize(2000)
    series = sim.run(150_000)
    _agrees_with_enumeration(dos, beta, series, {"E": lambda e, order: e,
                                                 "m2": lambda e, order: (order / sites**2 - 1.0) / (q - 1.0)})
    final = sim.state
    assert sim.running["energy"] == Potts(square(4, 2), q).bond_energy(final)
    np.testing.assert_array_equal(sim.running["counts"], np.bincount(final, minlength=q))


def test_ising_chain_matches_enumeration(cuda):
    dos = JointDOS("ising_dos_chain8")
    beta = 0.7
    with pytest.raises(ValueError, match="not ergodic"):
        Simulation(Ising(chain(8)), beta, "metropolis", seed=3)
    sim = Simulation(Ising(chain(8)), beta, "heatbath", seed=3)
    sim.thermalize(1000)
    _agrees_with_enumeration(dos, beta, sim.run(150_000), {"E": lambda e, mag: e})


def test_msc_ising_matches_kaufman(cuda):
    """Multi-spin-coded chain on a 64x4 torus against Kaufman's exact energy."""
    beta = 0.4
    sim = Simulation(Ising(square(64, 4)), beta, "metropolis", seed=5)
    sim.thermalize(1000)
    ts = sim.run(100_000)
    assert_consistent(ts["e"], kaufman_energy(beta, 64, 4))


@pytest.mark.parametrize("model", [Ising(square(6)), Potts(square(6), 3), Ising(square(64, 2))],
                         ids=["ising", "potts", "ising-msc"])
@pytest.mark.parametrize("chunk", [1, 7, 16, 50])
def test_streams_do_not_depend_on_the_chunk_size(cuda, model, chunk):
    """critmc tests/test_sim_chunks.py:7-16: the same streams whatever the chunk."""
    reference = Simulation(model, 0.6, "metropolis", seed=4).run(50)
    chunked = Simulation(model, 0.6, "metropolis", seed=4).run(50, chunk=chunk)
    assert list(chunked.raw) == list(reference.raw)
    for name, expected in reference.raw.items():
        got = chunked.raw[name]
        assert got.dtype == expected.dtype and np.array_equal(got, expected), name


def test_reproducible_given_seed(cuda):
    def energies():
        sim = Simulation(Potts(square(6), 4), 1.0, "heatbath+metropolis", seed=99)
        sim.thermalize(50)
        return sim.run(100)["E"]

    np.testing.assert_array_equal(energies(), energies())
