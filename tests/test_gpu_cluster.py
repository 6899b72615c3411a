"""Cluster updates (Swendsen-Wang, Wolff): bit-exact against the CPU replay on
both layouts, and critmc's exact results through Simulation schedules
(critmc tests/test_kernels.py:27-92 patterns with cluster moves)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch
from conftest import assert_consistent
from exact_helpers import JointDOS

import oracle
from critmc_b200 import Ising, Potts, Simulation, chain, hypercubic, square
from critmc_b200 import _lib
from critmc_b200.device import empty_bytes, ptr, stream_handle
from critmc_b200.layout import cb_pack, cb_unpack
from critmc_b200.models import _IsingMscChain

pytestmark = pytest.mark.gpu

WOLFF, SW = 3, 4

CASES = [
    ("ising", (18, 10), 0, 0.44),
    ("ising", (64, 32), 0, 0.44),  # bit layout
    ("ising", (64, 16, 8), 0, 0.22),  # bit layout, 3D
    ("ising", (6, 4, 8), 0, 0.25),
    ("ising", (16,), 0, 0.9),
    ("potts", (8, 6), 3, 1.0),
    ("potts", (4, 4, 4), 4, 0.5),
    ("potts", (64, 64), 10, 1.42),
]


@pytest.mark.parametrize("algo", [WOLFF, SW])
@pytest.mark.parametrize("kind,shape,q,beta", CASES)
def test_cluster_update_bit_identical_to_replay(cuda, kind, shape, q, beta, algo):
    lat = hypercubic(shape)
    model = Ising(lat) if kind == "ising" else Potts(lat, q)
    rng = np.random.default_rng(sum(shape) + algo)
    s0 = model.initial_state("random", rng)
    ch = model.to_device(s0, rng, cuda)
    bits = isinstance(ch, _IsingMscChain)
    dims = tuple(shape) + (1,) * (3 - len(shape))
    running = model.begin(s0)
    if kind == "ising":
        run_t = torch.tensor([[running["e_b"], running["m"]]], dtype=torch.int64, device=cuda)
        cnt_t = None
    else:
        run_t = torch.tensor([running["energy"]], dtype=torch.int64, device=cuda)
        cnt_t = torch.from_numpy(running["counts"].astype(np.int64)).to(cuda)
    stats = torch.zeros((1, 3), dtype=torch.int64, device=cuda)
    scratch = empty_bytes(_lib.lib().critmc_cluster_scratch_bytes(1, lat.n_sites), cuda)
    lay = np.ascontiguousarray(cb_pack(s0.astype(np.int8), shape))
    ref_stats = np.zeros(3, dtype=np.int64)
    e_ref, m_ref = (running["e_b"], running["m"]) if kind == "ising" else (running["energy"], 0)
    counts_ref = running["counts"].copy() if kind == "potts" else None
    spins = ch.words if bits else ch.spins
    for sweep in range(6):
        _lib.call("critmc_cluster_update", int(bits), ptr(spins), len(shape), *dims, q, 1, ch.key.ctypes.data,
                  beta, algo, sweep, ptr(run_t), ptr(cnt_t), ptr(stats), ptr(scratch), stream_handle(cuda))
        de, dm, cd, _ = oracle.cluster_update(lay, shape, q, ch.key, beta, algo, sweep, ref_stats)
        e_ref += de
        m_ref += dm
        if counts_ref is not None:
            counts_ref += cd
        got = ch.fetch()
        np.testing.assert_array_equal(got.astype(np.int8), cb_unpack(lay, shape).astype(np.int8))
        r = run_t.cpu().numpy().ravel()
        assert r[0] == e_ref
        if kind == "ising":
            assert r[1] == m_ref
        else:
            np.testing.assert_array_equal(cnt_t.cpu().numpy(), counts_ref)
        np.testing.assert_array_equal(stats.cpu().numpy().ravel(), ref_stats)
    # the running sums are those of the final configuration
    final = ch.fetch()
    if kind == "ising":
        assert r[0] == model.bond_energy(final) and r[1] == int(final.astype(np.int64).sum())
    else:
        assert r[0] == model.bond_energy(final)


@pytest.mark.parametrize("updates", ["sw", "wolff", "metropolis+sw", "heatbath+4*wolff"])
def test_ising_cluster_schedules_match_enumeration(cuda, updates):
    jd = JointDOS("ising_dos_square4")
    beta, n = 0.44, 16
    sim = Simulation(Ising(square(4)), beta, updates, seed=31)
    sim.thermalize(500)
    ts = sim.run(20_000)
    assert_consistent(ts["E"], jd.average(beta, lambda e, m: e))
    assert_consistent(ts["m2"], jd.average(beta, lambda e, m: (m / n) ** 2))
    state = sim.state
    assert sim.running["e_b"] == Ising(square(4)).bond_energy(state)
    if "wolff" in updates:
        assert ts.meta["mean_cluster"] > 1.0
    else:
        assert (ts["aux"][:, 3] >= 1).all()


@pytest.mark.parametrize("updates", ["sw", "wolff"])
def test_potts_cluster_schedules_match_enumeration(cuda, updates):
    jd = JointDOS("potts3_dos_square4x2")
    lat = square(4, 2)
    beta, q, n = 0.8, 3, 8
    sim = Simulation(Potts(lat, q), beta, updates, seed=41)
    sim.thermalize(500)
    ts = sim.run(20_000)
    assert_consistent(ts["E"], jd.average(beta, lambda e, s: e))
    assert_consistent(ts["m2"], jd.average(beta, lambda e, s: (s / n ** 2 - 1.0) / (q - 1.0)))
    state = sim.state
    np.testing.assert_array_equal(sim.running["counts"], np.bincount(state, minlength=q))


def test_auto_wolff_count_is_tuned(cuda):
    sim = Simulation(Ising(square(32)), 0.4406868, "wolff", seed=3)
    info = sim.thermalize(200)
    assert info["wolff_per_meas"] >= 1 and info["mean_cluster"] > 1
    assert "wolff_history" in info
