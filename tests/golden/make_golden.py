"""Generate the golden fixtures of the statistical parity tests from critmc itself.

Run in a container where the reference package is importable::

    PYTHONPATH=/path/to/critmc/src NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_golden.py

It writes ``tests/golden/critmc_exact.json``: exact results of critmc's own
exact layer (src/critmc/exact/kaufman.py, enumeration.py, chains.py,
onsager.py) on the lattices the GPU tests sample.  The tests read only the
JSON, so they run where critmc is absent.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from critmc import Potts, chain, square  # noqa: F401  (critmc must be on PYTHONPATH)
from critmc.exact import chains, dos, enumeration, kaufman, onsager, potts
from critmc.flathist import EnergyLevels, MucaResult, WangLandau, WLResult
from critmc.stats.autocorr import gamma_method
from scipy.optimize import brentq
from scipy.special import logsumexp

OUT = Path(__file__).resolve().parent / "critmc_exact.json"


def joint(jd) -> dict:
    return {
        "energies": jd.energies.tolist(),
        "orders": jd.orders.tolist(),
        "counts": jd.counts.tolist(),
        "n_sites": int(jd.n_sites),
    }


def ar1(seed: int, phi: float, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(n)
    x = np.empty(n)
    x[0] = e[0]
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    return x


def equal_height_beta(res, split: float, bracket) -> float:
    """beta at which the two maxima of the energy distribution from ln g are equal."""
    lv = res.levels
    v = res.visited
    e = lv.energies / lv.n_sites

    def f(b):
        a = np.where(v, res.ln_g - b * lv.energies, -np.inf)
        p = np.exp(a - logsumexp(a[v]))
        low = e < split
        return np.log(p[low].max()) - np.log(p[~low].max())

    return float(brentq(f, *bracket, xtol=1e-10))


def main() -> None:
    out: dict = {"source": "critmc 1.0.0 exact layer"}
    out["beta_c"] = float(onsager.BETA_C)
    betas = [0.30, 0.40, float(onsager.BETA_C), 0.48, 0.60]
    out["kaufman_energy"] = {
        str(L): {f"{b:.10f}": float(kaufman.energy(b, L)) for b in betas} for L in (16, 32, 64, 128)
    }
    out["kaufman_energy_rect"] = {
        f"{m}x{n}": {f"{b:.10f}": float(kaufman.energy(b, m, n)) for b in betas}
        for m, n in ((64, 2), (64, 4), (64, 6), (128, 8))
    }
    # Gamma-method results on seeded AR(1) series (regenerated from the seed in the tests)
    gam = []
    for seed, phi, n in ((1, 0.0, 4000), (2, 0.9, 20000), (3, 0.98, 50000)):
        x = ar1(seed, phi, n)
        r = gamma_method(x)
        gam.append({"seed": seed, "phi": phi, "n": n, "value": r.value, "error": r.error,
                    "tau_int": r.tau_int, "window": int(r.window)})
    out["gamma_method_ar1"] = gam
    out["ising_dos_square4"] = joint(enumeration.ising_joint_dos(square(4)))
    out["ising_dos_square4x2"] = joint(enumeration.ising_joint_dos(square(4, 2)))
    out["ising_dos_chain8"] = joint(enumeration.ising_joint_dos(chain(8)))
    out["potts3_dos_square4x2"] = joint(enumeration.potts_joint_dos(square(4, 2), 3))
    out["potts4_dos_square2"] = joint(enumeration.potts_joint_dos(square(2), 4))
    ring = {}
    for n in (2, 3):
        for beta in (0.7, 1.1):
            for N in (4, 8):
                ring[f"n{n}_N{N}_b{beta}"] = {
                    "energy": float(chains.on_ring_energy(beta, N, n)),
                    "specific_heat": float(chains.on_ring_specific_heat(beta, N, n)),
                }
    out["on_ring"] = ring
    # EA +-J couplings on a 4x4 torus and the energies of all 2^16 states
    rng = np.random.default_rng(20261203)
    lat = square(4)
    J = rng.choice([-1.0, 1.0], size=lat.n_bonds)
    e = enumeration.ea_energies(lat, J)
    out["ea_square4"] = {"couplings": J.tolist(), "energies_first_64": e[:64].tolist(),
                         "energy_sum": float(e.sum()), "energy_min": float(e.min())}
    # flat-histogram checks: exact g(E) of the 6x6 Ising torus (integers, as strings),
    # Kaufman energies at L = 6, the 3-state Potts joint DOS on the 4x3 torus and
    # the 10-state Potts transition point
    out["ising_dos_square6"] = {"g": [str(v) for v in dos.ising_dos(6).g]}
    out["kaufman_energy"]["6"] = {f"{b:.10f}": float(kaufman.energy(b, 6)) for b in (0.3, 0.44, 0.55, 0.6)}
    out["potts3_dos_square4x3"] = joint(enumeration.potts_joint_dos(square(4, 3), 3))
    out["potts_beta_c"] = {str(q): float(potts.beta_c(q)) for q in (3, 10)}
    # equal-height point of q = 10 Potts on the 8 x 8 torus, window [-1.95, -0.6],
    # split -1.3, from critmc's own Wang-Landau converged to ln f = 1e-6
    model, bc = Potts(square(8), 10), float(potts.beta_c(10))
    eq = [equal_height_beta(WangLandau(model, e_window=(-1.95, -0.6), seed=s).run(1e-6), -1.3, (bc - 0.2, bc + 0.1))
          for s in (1, 2, 3, 4)]
    out["potts10_L8_equal_height"] = {"beta": float(np.mean(eq)), "per_seed": eq, "ln_f_final": 1e-6,
                                      "window": [-1.95, -0.6], "split": -1.3}
    # critmc's analysis methods on a seeded synthetic multicanonical record
    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    from exact_helpers import synthetic_muca

    ln_g, idx, order, window, hist = synthetic_muca()
    lv = EnergyLevels("potts", 64, 128, 10)
    mu = MucaResult(lv, ln_g, idx, order, window, hist)
    ana: dict = {"canonical": {k: v.tolist() for k, v in mu.canonical([1.36, 1.40, 1.44]).items()},
                 "m2_head": mu.order_parameter_m2()[:8].tolist(),
                 "average_m2": mu.average(1.40, mu.order_parameter_m2())}
    for smooth in (0.0, 0.01):
        ana[f"p_smooth{smooth}"] = mu.energy_distribution(1.40, smooth)[1].tolist()
        ana[f"double_peak_smooth{smooth}"] = mu.double_peak(1.40, -1.3, smooth)
        ana[f"equal_height_smooth{smooth}"] = mu.equal_height_beta((1.2, 1.6), -1.3, smooth)
    ana["double_peak_auto_split"] = mu.double_peak(1.40)
    ana["phase_means"] = mu.phase_means(1.40, -1.3)
    ana["equal_weight"] = mu.equal_weight_beta((1.2, 1.6), -1.3)
    visited = hist > 0
    for win in (window, (0, lv.size - 1)):
        wl = WLResult(lv, np.where(visited, ln_g, 0.0), visited, win, 0, 0.0, 0.0)
        key = "wl_full" if win == (0, lv.size - 1) else "wl_window"
        ana[key] = {"normalized": np.where(visited, wl.normalized(), 0.0).tolist(),
                    "canonical": {k: v.tolist() for k, v in wl.canonical([1.36, 1.40]).items()}}
    out["flathist_analysis"] = ana
    # a series written by critmc itself (TimeSeries.save: .npz + JSON metadata),
    # read back by this project's loader in the format tests
    from critmc import Ising, Simulation

    sim = Simulation(Ising(square(4)), 0.44, "metropolis", seed=5)
    sim.thermalize(20)
    sim.run(200).save(OUT.parent / "critmc_series_ising4.npz")
    # critmc's Simulation host logic driven by a deterministic fake advance
    from critmc import ON as RefON
    from critmc import Ising as RefIsing
    from exact_helpers import SIM_SCENARIOS, fake_advance, summarize_series
    from critmc.io import to_jsonable as ref_jsonable

    def fake_model(kind):
        base = RefIsing if kind == "ising" else RefON
        args = (square(8),) if kind == "ising" else (square(8), 2)

        class Fake(base):
            calls: list = []

            def advance(self, state, running, beta, rng, schedule, n_meas, ws):
                Fake.calls.append([int(n_meas), schedule.tolist(), running.get("step")])
                return fake_advance(len(Fake.calls) - 1, schedule, n_meas, self.n_sites, kind)

        Fake.calls = []
        return Fake(*args), Fake

    sims = []
    for kind, updates, therm, n_chunks, n_run, chunk in SIM_SCENARIOS:
        model, cls = fake_model(kind)
        sim = Simulation(model, 0.5, updates, seed=11)
        tuning = sim.thermalize(therm, n_chunks=n_chunks)
        ts = sim.run(n_run, chunk=chunk)
        sims.append(ref_jsonable({"calls": cls.calls, "tuning": tuning, "final_tuning": sim.tuning(),
                                  "series": summarize_series(ts.raw, ts.meta), "n_therm": sim.n_therm,
                                  "n_meas": sim.n_meas}))
    out["simulation_host_logic"] = sims

    # model host methods of critmc: seeded initial states, energies, metadata, derived observables
    from critmc import cubic
    from critmc.models import derive as ref_derive
    from critmc.rng import make_rng as ref_make_rng

    models = {"ising": RefIsing(square(6), h=0.25), "potts": Potts(cubic(4), 5), "on": RefON(chain(8), 3)}
    host: dict = {}
    for name, mdl in models.items():
        s0 = mdl.initial_state("random", ref_make_rng(3, "start"))
        s1 = mdl.initial_state("ordered", ref_make_rng(3))
        host[name] = {"random": np.asarray(s0, dtype=np.float64).ravel().tolist(),
                      "ordered": np.asarray(s1, dtype=np.float64).ravel().tolist(),
                      "energy_random": float(mdl.energy(s0)), "meta": mdl.meta(), "spec": mdl.spec()}
    rng = np.random.default_rng(99)
    raws = {"ising": ({"E": rng.integers(-72, 72, 20).astype(float), "M": rng.integers(-36, 37, 20)},
                      {"model": "ising", "N": 36}),
            "potts": ({"E": rng.integers(-192, 0, 20).astype(float), "counts": rng.multinomial(64, [0.2] * 5, 20)},
                      {"model": "potts", "N": 64, "q": 5}),
            "on": ({"E": rng.normal(size=20), "M": rng.normal(size=(20, 3)) * 3}, {"model": "on", "N": 8})}
    for name, (raw, meta) in raws.items():
        host[name]["derive"] = {k: np.asarray(v).tolist() for k, v in ref_derive(raw, meta).items()}
    out["model_host"] = host

    # critmc's lattice tables and keyed random streams (interfaces kept exactly)
    from critmc import hypercubic as ref_hypercubic
    from critmc import triangular as ref_triangular
    from critmc.lattice import make_lattice as ref_make_lattice
    from critmc.rng import spawn_rngs as ref_spawn

    lats = {"chain6": chain(6), "square4x3": square(4, 3), "cubic3": ref_make_lattice("cubic", 3),
            "hyper2x2x2x2": ref_hypercubic((2, 2, 2, 2)), "triangular4": ref_triangular(4),
            "square_named": ref_make_lattice("square", 5)}
    out["lattices"] = {
        k: {"name": v.name, "shape": list(v.shape), "nbr": v.nbr.tolist(), "bonds": v.bonds.tolist(),
            "bond_axis": v.bond_axis.tolist(), "coords": v.coords.tolist(),
            "positions": np.asarray(v.positions).tolist(), "primitive": np.asarray(v.primitive).tolist(),
            "sublattice": None if v.sublattice is None else v.sublattice.tolist(), "z": int(v.z),
            "site_ones": int(v.site(*([1] * v.dim))),
            "kmin": v.kmin(0).tolist()} for k, v in lats.items()}
    streams = {}
    for label, args in (("int", (5,)), ("int_keys", (5, "ising", 64, 2)), ("str_key", (123, "walker", 7)),
                        ("tuple_key", (9, (1, 2))), ("bool_key", (4, True, False)), ("float_key", (4, 0.5)),
                        ("seedseq", (np.random.SeedSequence(77),)), ("seedseq_keys", (np.random.SeedSequence(77), 3))):
        streams[label] = ref_make_rng(*args).integers(0, 2**32, size=4).tolist()
    streams["spawn"] = [g.integers(0, 2**32, size=2).tolist() for g in ref_spawn(8, 3, "x")]
    out["rng_streams"] = streams

    # critmc's EA +-J couplings for a seed, its temperature ladder and a sample energy
    from critmc.glass import EdwardsAnderson as RefEA
    from critmc.glass import geometric_temperatures as ref_temps

    ea = {}
    for sd in (1, 2):
        sample = RefEA(cubic(4), disorder="bimodal", seed=sd)
        state = np.where(np.random.default_rng(sd).random(64) < 0.5, -1, 1)
        ea[str(sd)] = {"couplings": sample.couplings.tolist(), "energy": float(sample.energy(state))}
    out["ea_samples"] = {"cubic4": ea, "temperatures": ref_temps(0.5, 2.0, 32).tolist()}
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
