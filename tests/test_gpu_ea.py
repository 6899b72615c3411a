"""Spin-glass parallel tempering on the GPU: bit-exact against the CPU replay and
against exact enumeration (critmc tests/test_glass.py)."""

from __future__ import annotations

import numpy as np
import pytest
from exact_helpers import ea_exact, golden

import oracle
from critmc_b200 import cubic, square
from critmc_b200.glass import (EdwardsAnderson, ParallelTempering, SpinGlassCampaign,
                               geometric_temperatures)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lat,m,n_bins,sps", [
    (square(4), 8, 7, 1),
    (cubic(4), 16, 6, 2),
    (cubic(6), 32, 5, 1),
    (square(8), 5, 6, 1),
])
def test_campaign_bit_identical_to_replay(cuda, lat, m, n_bins, sps):
    samples = [EdwardsAnderson(lat, disorder="bimodal", seed=10 + i) for i in range(3)]
    temps = geometric_temperatures(0.5, 2.0, m)
    camp = SpinGlassCampaign(samples, temps, seeds=[100 + i for i in range(3)], sweeps_per_step=sps,
                             device=cuda)
    runs = camp.run(n_bins)
    runs2 = camp.run(3)  # a second call continues the streams (step counter)
    gpu_spins = camp.spins()
    conf = camp.conf_at.cpu().numpy()
    labels = camp.labels.cpu().numpy()
    for i in range(3):
        spins = camp.initial_spins[i].copy()
        perm = np.tile(np.arange(m, dtype=np.int32), (2, 1))
        lab = np.zeros((2, m), dtype=np.int32)
        table = camp.swap_thr.cpu().numpy().view(np.uint32)
        out1 = oracle.ea_pt_run(spins, samples[i].couplings, lat.shape, camp.keys[i], camp.betas, table,
                                perm, lab, n_steps=(1 << n_bins) - 1, n_bins=n_bins, sweeps_per_step=sps)
        out2 = oracle.ea_pt_run(spins, samples[i].couplings, lat.shape, camp.keys[i], camp.betas, table,
                                perm, lab, n_steps=7, n_bins=3, t0=(1 << n_bins) - 1,
                                sweeps_per_step=sps)
        np.testing.assert_array_equal(runs[i].acc, out1[0])
        np.testing.assert_array_equal(runs2[i].acc, out2[0])
        np.testing.assert_array_equal(runs[i].label_hist, out1[3])
        np.testing.assert_array_equal(runs[i].trips, out1[4])
        with np.errstate(invalid="ignore", divide="ignore"):
            np.testing.assert_array_equal(runs[i].swap_rate, out1[1] / out1[2])
        np.testing.assert_array_equal(conf[i], perm)
        np.testing.assert_array_equal(labels[i], lab)
        for r in range(2):
            for k in range(m):
                np.testing.assert_array_equal(gpu_spins[i, r, k], spins[r, perm[r, k]])


def test_parallel_tempering_matches_enumeration(cuda):
    """critmc tests/test_glass.py:26-52 with +-J couplings on a 4x4 torus."""
    lat = square(4)
    J = np.asarray(golden()["ea_square4"]["couplings"])
    ea = EdwardsAnderson(lat, J)
    temps = geometric_temperatures(0.4, 2.5, 8)
    run = ParallelTempering(ea, temps, seed=5, device=cuda).run(16)
    eq = run.equilibrium()
    ex = ea_exact(lat, J, run.temperatures)
    np.testing.assert_allclose(eq["e"], ex["e"], atol=0.01)
    np.testing.assert_allclose(eq["q2"], ex["q2"], atol=0.01)
    np.testing.assert_allclose(eq["ql"], ex["ql"], atol=0.01)
    assert np.all(run.swap_rate > 0.3)
    assert run.trips.sum() > 100


def test_same_seed_same_couplings_and_spins_as_critmc_convention(cuda):
    """Couplings come from make_rng(seed).choice([-1, 1]) as in critmc glass.py:62-63."""
    from critmc_b200.rng import make_rng

    lat = cubic(4)
    ea = EdwardsAnderson(lat, disorder="bimodal", seed=77)
    np.testing.assert_array_equal(ea.couplings, make_rng(77).choice([-1.0, 1.0], size=lat.n_bonds))
    with pytest.raises(ValueError):
        EdwardsAnderson(lat, disorder="gaussian", seed=1)


def _campaigns(sizes, temps, n_samples, cuda, sps=1):
    out = []
    for L in sizes:
        lat = cubic(L)
        samples = [EdwardsAnderson(lat, disorder="bimodal", seed=1000 * L + i) for i in range(n_samples)]
        out.append(SpinGlassCampaign(samples, temps, seeds=[7000 * L + i for i in range(n_samples)],
                                     sweeps_per_step=sps, device=cuda))
    return out


def test_multi_size_campaign_equals_per_size_runs(cuda):
    """Uneven sizes in one persistent launch give each size's own results, over two calls."""
    from critmc_b200.glass import MultiSizeCampaign

    temps = geometric_temperatures(0.5, 2.0, 32)
    sizes = (4, 6, 8, 10, 12, 16)
    alone = _campaigns(sizes, temps, 5, cuda)
    mixed = MultiSizeCampaign(_campaigns(sizes, temps, 5, cuda))
    for n_bins in (5, 3):
        want = [c.run(n_bins) for c in alone]
        got = mixed.run(n_bins)
        for runs_a, runs_b in zip(want, got):
            for a, b in zip(runs_a, runs_b):
                np.testing.assert_array_equal(a.acc, b.acc)
                np.testing.assert_array_equal(a.swap_rate, b.swap_rate)
                np.testing.assert_array_equal(a.label_hist, b.label_hist)
                np.testing.assert_array_equal(a.trips, b.trips)
    for ca, cb in zip(alone, mixed.campaigns):
        np.testing.assert_array_equal(ca.spins(), cb.spins())
