"""Cluster updates (Swendsen-Wang, Wolff): bit-exact against the CPU replay on
both Ising layouts, Potts and the O(n) models, and critmc's exact results
through Simulation schedules (critmc tests/test_kernels.py:27-109 patterns with
cluster moves)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch
from conftest import assert_consistent
from exact_helpers import JointDOS

import oracle
from critmc_b200 import ON, Ising, Potts, Simulation, chain, hypercubic, square
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
    for name, fn in {"E": lambda e, mag: e, "m2": lambda e, mag: np.square(mag / n)}.items():
        assert_consistent(ts[name], jd.average(beta, fn))
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
    for name, fn in {"E": lambda e, order: e, "m2": lambda e, order: (order / n**2 - 1.0) / (q - 1.0)}.items():
        assert_consistent(ts[name], jd.average(beta, fn))
    state = sim.state
    np.testing.assert_array_equal(sim.running["counts"], np.bincount(state, minlength=q))


def test_auto_wolff_count_is_tuned(cuda):
    sim = Simulation(Ising(square(32)), 0.4406868, "wolff", seed=3)
    info = sim.thermalize(200)
    assert info["wolff_per_meas"] >= 1 and info["mean_cluster"] > 1
    assert "wolff_history" in info


ON_CASES = [
    ((16, 8), 2, 0.9),
    ((64, 32), 2, 1.1),
    ((16,), 2, 1.1),
    ((8, 8, 4), 3, 0.7),
    ((6, 4), 3, 1.5),
]


@pytest.mark.parametrize("algo", [WOLFF, SW])
@pytest.mark.parametrize("shape,n,beta", ON_CASES)
def test_on_cluster_update_bit_identical_to_replay(cuda, shape, n, beta, algo):
    """Embedded-Ising reflections (critmc kernels/on.py:265-345) against the CPU replay."""
    lat = hypercubic(shape)
    model = ON(lat, n)
    rng = np.random.default_rng(sum(shape) + 10 * n + algo)
    s0 = model.initial_state("random", rng)
    ch = model.to_device(s0, rng, cuda)
    dims = tuple(shape) + (1,) * (3 - len(shape))
    comps = np.ascontiguousarray(np.stack([cb_pack(s0[:, k].astype(np.float32), shape) for k in range(n)]))
    comps = comps.reshape(n, -1)
    stats = torch.zeros((1, 3), dtype=torch.int64, device=cuda)
    scratch = empty_bytes(_lib.lib().critmc_cluster_scratch_bytes(1, lat.n_sites), cuda)
    ref_stats = np.zeros(3, dtype=np.int64)
    for sweep in range(6):
        _lib.call("critmc_on_cluster_update", ptr(ch.spins), len(shape), *dims, n, 1, ch.key.ctypes.data, beta, algo,
                  sweep, ptr(stats), ptr(scratch), stream_handle(cuda))
        oracle.on_cluster_update(comps, shape, ch.key, beta, algo, sweep, ref_stats)
        got = ch.spins.cpu().numpy().reshape(n, -1)
        assert np.array_equal(got.view(np.uint32), comps.view(np.uint32))
        np.testing.assert_array_equal(stats.cpu().numpy().ravel(), ref_stats)
    # reflections keep unit length up to rounding
    assert np.allclose(np.linalg.norm(ch.fetch(), axis=1), 1.0, atol=1e-5)
    if algo == WOLFF:
        assert ref_stats[0] > 0


def test_on_mixed_cluster_schedule_matches_replay(cuda):
    """heatbath + overrelax + wolff + sw per measurement: E, M and spins bit for bit."""
    shape, n, beta = (16, 16), 2, 1.0
    model = ON(hypercubic(shape), n)
    rng = np.random.default_rng(77)
    s0 = model.initial_state("random", rng)
    ch = model.to_device(s0, rng, cuda)
    key = ch.key.copy()
    sched = np.array([[2, 1], [5, 2], [3, 3], [4, 1]])
    running = model.begin(s0)
    out = model.advance(ch, running, beta, sched, 5)
    # replay: sweep rows through oracle.on_run (ending in a measurement), cluster rows through the oracle
    s = s0.astype(np.float32)
    sweep = 0
    ref_e, ref_aux = [], []
    for _ in range(5):
        _, _, _, _, aux1 = oracle.on_run(s, shape, n, key, beta, 1.0, sched[:2], 1, sweep0=sweep)
        sweep += 3
        comps = np.ascontiguousarray(np.stack([cb_pack(s[:, k], shape) for k in range(n)])).reshape(n, -1)
        st = np.zeros(3, dtype=np.int64)
        for code, reps in sched[2:]:
            for _ in range(reps):
                oracle.on_cluster_update(comps, shape, key, beta, int(code), sweep, st)
                sweep += 1
        s = np.ascontiguousarray(np.stack([cb_unpack(comps[k], shape) for k in range(n)], axis=1))
        e, _, _, _, aux2 = oracle.on_run(s, shape, n, key, beta, 1.0, [[5, 0]], 1, sweep0=sweep)
        ref_e.append(e[0])
        ref_aux.append([aux1[0][0] + aux2[0][0], st[0], st[1], st[2]])
    np.testing.assert_array_equal(out["E"], ref_e)
    np.testing.assert_array_equal(out["aux"], np.array(ref_aux))
    assert np.array_equal(ch.fetch().astype(np.float32), s)


@pytest.mark.parametrize("n_comp", [2, 3])
@pytest.mark.parametrize("updates", ["3*wolff", "heatbath+sw"])
def test_on_cluster_ring_matches_transfer_operator(cuda, n_comp, updates):
    """critmc tests/test_kernels.py:95-109 with cluster moves."""
    from exact_helpers import golden

    ref = golden()["on_ring"][f"n{n_comp}_N8_b1.1"]
    beta, n_sites = 1.1, 8
    sim = Simulation(ON(chain(n_sites), n_comp), beta, updates, seed=6)
    sim.thermalize(1000)
    ts = sim.run(30_000)
    assert_consistent(ts["e"], ref["energy"])
    e = ts["E"]
    assert beta ** 2 * e.var() / n_sites == pytest.approx(ref["specific_heat"], rel=0.1)
    s = sim.state
    assert np.allclose(np.linalg.norm(s, axis=1), 1.0, atol=1e-6)
