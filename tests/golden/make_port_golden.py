"""Fixtures that pin the C port of critmc's CPU Ising kernel (oracle/oracle_critmc_port.c).

Run where the reference package is importable::

    PYTHONPATH=/path/to/critmc/src NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_port_golden.py

For a few seeded critmc ``Simulation`` runs it records the initial spins, the
Generator (PCG64DXSM) state handed to the kernel, and critmc's series and final
spins; plus raw outputs of PCG64DXSM from numpy for a seed.  Writes
``tests/golden/critmc_port.json``; the tests read only the JSON.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from critmc import Ising, Simulation, hypercubic  # critmc must be on PYTHONPATH

OUT = Path(__file__).resolve().parent / "critmc_port.json"

CASES = [
    # shape, h, beta, updates, seed, n_meas
    ((16, 16), 0.0, 0.4406868, "metropolis", 3, 20),
    ((16, 12), 0.2, 0.40, "heatbath+2*metropolis", 4, 10),
    ((6, 6, 6), 0.0, 0.2216546, "metropolis", 5, 8),
    ((32, 32), -0.1, 0.5, "heatbath", 6, 6),
]


def main() -> None:
    out = {"cases": []}
    for shape, h, beta, updates, seed, n_meas in CASES:
        sim = Simulation(Ising(hypercubic(shape), h), beta, updates, seed=seed)
        start = sim.state.copy()
        gen = sim.rng.bit_generator.state["state"]
        ts = sim.run(n_meas)
        out["cases"].append({
            "shape": list(shape), "h": h, "beta": beta, "updates": updates, "seed": seed, "n_meas": n_meas,
            "schedule": sim.schedule.tolist(), "start": start.astype(int).tolist(),
            "pcg_state": str(gen["state"]), "pcg_inc": str(gen["inc"]),
            "Eb": ts.raw["Eb"].tolist(), "M": ts.raw["M"].tolist(), "aux": ts.raw["aux"].tolist(),
            "final": sim.state.astype(int).tolist(),
        })
    bg = np.random.PCG64DXSM(20261204)
    st = bg.state["state"]
    out["pcg_raw"] = {"state": str(st["state"]), "inc": str(st["inc"]),
                      "outputs": [str(int(x)) for x in bg.random_raw(64)]}
    OUT.write_text(json.dumps(out) + "\n")


if __name__ == "__main__":
    main()
