"""Statistical acceptance on the plain configuration: 2D Ising on the 32 x 32
torus at beta_c = ln(1 + sqrt 2) / 2, int8 spins from a hot start, checkerboard
Metropolis, 2,000 thermalisation sweeps then 50,000 measured sweeps per seed.

For every seed, the Gamma-method mean of the energy per site and its error give
the pull (mean - Kaufman) / error against Kaufman's exact finite-torus energy;
over many independent seeds the pulls must average to zero within 0.3 and have
a standard deviation in [0.8, 1.2].  This is critmc's validation method
(experiments/e01_validation.py:25-43, 67-106; exact/kaufman.py:152-156;
stats/calibration.py:130-227), with Kaufman's value from the fixture that
critmc's own exact layer wrote.

The seeds run as one batched call of the byte-lattice entry point.  Each chain
is built exactly as ``Simulation(Ising(square(32)), beta, updates, seed=s)``
builds it (the same Generator draws for the start and the Philox key), and the
first test checks that one chain of the batch is bit-identical to that
Simulation, so the batch is the same set of chains that seeded Simulations
would give.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from critmc_b200 import Ising, Simulation, _lib, square
from critmc_b200.device import ptr, stream_handle, to_dev, to_host
from critmc_b200.layout import cb_pack
from critmc_b200.models import HEATBATH, METROPOLIS
from critmc_b200.rng import make_rng, philox_key
from exact_helpers import beta_c, kaufman_energy, pulls

pytestmark = pytest.mark.gpu

L = 32
N_THERM, N_MEAS = 2_000, 50_000
SEEDS = list(range(1000, 1128))  # 128 independent seeds (at least 64 asked for)


def _seeded_batch(cuda, seeds, beta, code, n_therm, n_meas):
    """E_b series (n_seeds, n_meas) of the seeded chains after n_therm discarded sweeps."""
    model = Ising(square(L))
    states, keys = [], []
    for s in seeds:
        rng = make_rng(s)  # Simulation: rng = make_rng(seed); start, then the chain's key
        states.append(model.initial_state("random", rng))
        keys.append(philox_key(rng))
    n = len(seeds)
    keys = np.ascontiguousarray(np.stack(keys), dtype=np.uint32)
    tables = np.ascontiguousarray(model.tables(beta)[0][None])
    spins = to_dev(np.stack([cb_pack(s, (L, L)) for s in states]), cuda)
    running = torch.from_numpy(np.array([[model.bond_energy(s), int(s.astype(np.int64).sum())]
                                         for s in states], np.int64)).to(cuda)
    sched = np.array([[code, 1]], np.int64)
    out = None
    sweep = 0
    for count in (n_therm, n_meas):
        if count == 0:
            continue
        e = torch.empty((n, count), dtype=torch.int64, device=cuda)
        m = torch.empty_like(e)
        aux = torch.empty((n, count, 4), dtype=torch.int64, device=cuda)
        _lib.call_on(cuda, "critmc_ising_byte_run", ptr(spins), 2, L, L, 1, n, keys.ctypes.data, tables.ctypes.data,
                     1, sweep, sched.ctypes.data, 1, count, ptr(running), ptr(e), ptr(m), ptr(aux),
                     stream_handle(cuda))
        sweep += count
        out = to_host(e)
    return out


def test_batched_chain_is_the_seeded_simulation(cuda):
    beta = beta_c()
    sim = Simulation(Ising(square(L)), beta, "metropolis", seed=SEEDS[1], device=cuda)
    alone = sim.run(300).raw["Eb"]
    batch = _seeded_batch(cuda, SEEDS[:3], beta, METROPOLIS, 0, 300)
    np.testing.assert_array_equal(alone, batch[1])


@pytest.mark.parametrize("update,code", [("metropolis", METROPOLIS), ("heatbath", HEATBATH)])
def test_kaufman_pulls_32x32_at_beta_c(cuda, update, code):
    beta = beta_c()
    exact = kaufman_energy(beta, L)
    eb = _seeded_batch(cuda, SEEDS, beta, code, N_THERM, N_MEAS)
    e = eb.astype(np.float64) / (L * L)  # energy per site (h = 0)
    p = pulls(list(e), exact)
    mean, sd = float(p.mean()), float(p.std(ddof=1))
    print(f"\n{update}: {len(SEEDS)} seeds, pulls mean {mean:+.3f} sd {sd:.3f}, "
          f"<e> {e.mean():.6f} vs Kaufman {exact:.6f}")
    assert abs(mean) < 0.3, f"{update}: mean pull {mean:+.3f} (sd {sd:.3f})"
    assert 0.8 <= sd <= 1.2, f"{update}: pull sd {sd:.3f} (mean {mean:+.3f})"
