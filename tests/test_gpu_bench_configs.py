"""Bit-exact replay of the configurations the benchmark times.

The benchmark's numbers are only worth quoting if the kernels produce the
oracle's bits at those very shapes, launch shapes and batch sizes:

- 2D Ising, multi-spin coded, L = 4096, beta in {0.40, beta_c, 0.48} x 64
  chains (192 chains in three acceptance-table groups), at the launch shape the
  autotuner picks on a B200 (32 rows per thread, 8 inline planes, one launch
  per half-sweep) and at the library's default shape; L = 1024 with the same
  betas and batch.  Three chains, one per beta group, are replayed by the
  oracle (critmc kernels/ising.py:174-237 restated) for Metropolis and then heat
  bath sweeps.
- 3D Edwards-Anderson +-J, the multi-size campaign of L in {6, 8, 10, 12, 16}
  in one persistent launch; one L = 16 and one L = 12 sample are replayed
  (critmc kernels/glass.py:81-163 restated) for 31 steps.
- O(n): XY and Heisenberg ensembles of 128 chains at L = 256 (updated in HBM,
  not shared memory), 1 heat bath + 4 over-relaxation per step, 2 steps; one
  chain of each is replayed (critmc kernels/on.py:141-261, 349-418 restated).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from critmc_b200 import ON, cubic, hypercubic
from critmc_b200.autotune import msc_mode
from critmc_b200.ensemble import IsingEnsemble
from critmc_b200.glass import EdwardsAnderson, MultiSizeCampaign, SpinGlassCampaign, geometric_temperatures
from critmc_b200.on_models import ONEnsemble

pytestmark = pytest.mark.gpu

BETAS = (0.40, 0.4406868, 0.48)


def _replay_ising_ensemble(ens: IsingEnsemble, chains, n_met: int, n_hb: int) -> None:
    starts = {c: ens.state(c).astype(np.int8) for c in chains}
    met = ens.run(n_met, "metropolis", host=True)
    met = {k: getattr(met, k).numpy().copy() for k in ("Eb", "M", "aux")}
    hb = ens.run(n_hb, "heatbath", host=True)
    hb = {k: getattr(hb, k).numpy().copy() for k in ("Eb", "M", "aux")}
    for c in chains:
        beta = ens.betas[c // ens.chains_per_beta]
        s = np.ascontiguousarray(starts[c])
        e, m, aux, run = oracle.ising_msc_run(s, ens.shape, ens.keys[c], beta, 0.0, [[0, 1]], n_met)
        np.testing.assert_array_equal(met["Eb"][c], e, err_msg=f"chain {c} Metropolis E_b")
        np.testing.assert_array_equal(met["M"][c], m, err_msg=f"chain {c} Metropolis M")
        np.testing.assert_array_equal(met["aux"][c], aux, err_msg=f"chain {c} Metropolis aux")
        e, m, aux, run = oracle.ising_msc_run(s, ens.shape, ens.keys[c], beta, 0.0, [[2, 1]], n_hb,
                                              sweep0=n_met, running=run)
        np.testing.assert_array_equal(hb["Eb"][c], e, err_msg=f"chain {c} heat bath E_b")
        np.testing.assert_array_equal(hb["M"][c], m, err_msg=f"chain {c} heat bath M")
        np.testing.assert_array_equal(hb["aux"][c], aux, err_msg=f"chain {c} heat bath aux")
        np.testing.assert_array_equal(ens.state(c), s, err_msg=f"chain {c} spins")


@pytest.mark.parametrize("mode,k_inline", [(msc_mode(32, 1), 8), (0, 4)])
def test_msc_L4096_benchmark_batch_replays(cuda, mode, k_inline):
    ens = IsingEnsemble(4096, BETAS, 64, seed=1000, device=cuda, mode=mode, k_inline=k_inline)
    _replay_ising_ensemble(ens, (0, 64, 191), 3, 3)


def test_msc_L1024_benchmark_batch_replays(cuda):
    ens = IsingEnsemble(1024, BETAS, 64, seed=8, device=cuda)
    _replay_ising_ensemble(ens, (0, 100, 191), 8, 8)


def test_ea_multi_size_campaign_replays_largest_sizes(cuda):
    temps = geometric_temperatures(0.5, 2.0, 32)
    n_samples = 16
    camps, samples = [], {}
    for L in (6, 8, 10, 12, 16):
        ss = [EdwardsAnderson(cubic(L), disorder="bimodal", seed=L * 100000 + i) for i in range(n_samples)]
        samples[L] = ss
        camps.append(SpinGlassCampaign(ss, temps, seeds=[L * 200000 + i for i in range(n_samples)], device=cuda))
    mc = MultiSizeCampaign(camps)
    n_bins = 5
    runs = mc.run(n_bins)  # 31 steps, every size in one persistent launch
    for L, i in ((16, 3), (12, 11)):
        j = (6, 8, 10, 12, 16).index(L)
        camp = mc.campaigns[j]
        m = len(temps)
        spins = camp.initial_spins[i].copy()
        perm = np.tile(np.arange(m, dtype=np.int32), (2, 1))
        lab = np.zeros((2, m), dtype=np.int32)
        table = camp.swap_thr.cpu().numpy().view(np.uint32)
        acc, swap_acc, swap_try, label_hist, trips = oracle.ea_pt_run(
            spins, samples[L][i].couplings, (L, L, L), camp.keys[i], camp.betas, table, perm, lab,
            n_steps=(1 << n_bins) - 1, n_bins=n_bins)
        got = runs[j][i]
        np.testing.assert_array_equal(got.acc, acc, err_msg=f"L={L} sample {i} acc")
        np.testing.assert_array_equal(got.label_hist, label_hist)
        np.testing.assert_array_equal(got.trips, trips)
        with np.errstate(invalid="ignore", divide="ignore"):
            np.testing.assert_array_equal(got.swap_rate, swap_acc / swap_try)
        np.testing.assert_array_equal(camp.conf_at.cpu().numpy()[i], perm)
        gpu_spins = camp.spins()
        for r in range(2):
            for k in range(m):
                np.testing.assert_array_equal(gpu_spins[i, r, k], spins[r, perm[r, k]])


@pytest.mark.parametrize("n", [2, 3])
def test_on_L256_ensemble_replays(cuda, n):
    temps = np.linspace(0.7, 1.1, 16)
    sched = np.array([[2, 1], [5, 4]])
    ens = ONEnsemble(ON(hypercubic((256, 256)), n), temps, 8, seed=256, device=cuda)
    chains = (0, 77)
    starts = {c: ens.chain(c).astype(np.float32) for c in chains}
    out = ens.run(2, sched)
    got = {k: v.cpu().numpy() for k, v in out.items()}
    for c in chains:
        t = c // ens.chains_per_temperature
        s = np.ascontiguousarray(starts[c])
        e, m, sc, ss, aux = oracle.on_run(s, (256, 256), n, ens.keys[c], float(ens.betas[t]), float(ens.steps[t]),
                                          sched, 2)
        np.testing.assert_array_equal(got["E"][c], e)
        np.testing.assert_array_equal(got["M"][c], m)
        np.testing.assert_array_equal(got["stiff_c"][c], sc)
        np.testing.assert_array_equal(got["stiff_s"][c], ss)
        np.testing.assert_array_equal(got["aux"][c], aux)
        np.testing.assert_array_equal(ens.chain(c).astype(np.float32), s)
