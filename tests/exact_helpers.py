"""Exact references for the statistical tests, read from ``golden/critmc_exact.json``.

The fixture holds outputs of critmc's own exact layer (generated by
``golden/make_golden.py``).  This module only evaluates canonical averages
from the stored densities of states and restates Wolff's Gamma-method
(critmc src/critmc/stats/autocorr.py:363-516, single primary observable,
S = 1.5) for error bars of autocorrelated series.
"""

from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "critmc_exact.json"


@lru_cache(maxsize=1)
def golden() -> dict:
    return json.loads(GOLDEN.read_text())


def kaufman_energy(beta: float, L: int, M: int | None = None) -> float:
    """Kaufman's exact energy per site of the L x M torus at a tabulated beta."""
    g = golden()
    table = g["kaufman_energy"][str(L)] if M is None or M == L else g["kaufman_energy_rect"][f"{L}x{M}"]
    return float(table[f"{beta:.10f}"])


def beta_c() -> float:
    return float(golden()["beta_c"])


class JointDOS:
    """Exact joint density of states g(E, O) from the fixture."""

    def __init__(self, name: str):
        d = golden()[name]
        self.energies = np.asarray(d["energies"], dtype=np.float64)
        self.orders = np.asarray(d["orders"], dtype=np.float64)
        self.counts = np.asarray(d["counts"], dtype=np.float64)
        self.n_sites = int(d["n_sites"])

    def average(self, beta: float, fn, h: float = 0.0) -> float:
        """Canonical average of fn(E, O) at ``beta`` (field ``h`` coupling to O)."""
        energy = self.energies[:, None] + 0.0 * self.orders[None, :]
        order = self.orders[None, :] + 0.0 * self.energies[:, None]
        filled = self.counts > 0
        log_w = np.full(self.counts.shape, -np.inf)
        log_w[filled] = np.log(self.counts[filled]) - beta * (energy[filled] - h * order[filled])
        prob = np.exp(log_w - log_w[filled].max())
        return float((prob * fn(energy, order)).sum() / prob.sum())


def gamma_error(x: np.ndarray, S: float = 1.5) -> tuple[float, float, float]:
    """(mean, error, tau_int) of a single series by Wolff's automatic windowing."""
    x = np.asarray(x, dtype=np.float64)
    n = x.size
    mean = float(x.mean())
    d = x - mean
    if np.ptp(x) == 0:
        return mean, 0.0, 0.5
    t_max = n // 2
    nfft = 1 << (2 * n - 1).bit_length()
    spec = np.fft.rfft(d, n=nfft)
    gam = np.fft.irfft(spec.real ** 2 + spec.imag ** 2, n=nfft)[: t_max + 1]
    gam /= n - np.arange(t_max + 1)
    # Wolff's window: the first W at which exp(-W / tau(W)) - tau(W) / sqrt(W N) turns
    # negative, with tau(W) = S / ln(1 + 1 / G(W)) and G(W) = sum_{t<=W} Gamma(t) / Gamma(0)
    windows = np.arange(1, gam.size)
    summed = np.cumsum(gam[1:]) / gam[0]
    tau = np.full(windows.size, 1e-300)
    positive = summed > 0
    with np.errstate(divide="ignore", over="ignore"):
        tau[positive] = S / np.log1p(np.reciprocal(summed[positive]))
    tau = np.maximum(tau, 1e-300)
    criterion = np.exp(-windows / tau) - tau / np.sqrt(windows * float(n))
    below = np.flatnonzero(criterion < 0)
    w_opt = int(windows[below[0]] if below.size else windows[-1])
    c_f = gam[0] + 2.0 * gam[1:w_opt + 1].sum()
    gam = gam + c_f / n  # bias of the subtracted mean
    c_f = gam[0] + 2.0 * gam[1:w_opt + 1].sum()
    tau = c_f / (2.0 * gam[0])
    return mean, float(np.sqrt(c_f / n)) if c_f > 0 else float("nan"), float(tau)


def ar1(seed: int, phi: float, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(n)
    x = np.empty(n)
    x[0] = e[0]
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    return x


def pulls(series: list[np.ndarray], exact: float) -> np.ndarray:
    """(Gamma-method mean - exact) / error for each independent chain."""
    out = []
    for x in series:
        m, err, _ = gamma_error(x)
        out.append((m - exact) / err)
    return np.asarray(out)


def ea_exact(lattice, couplings, temperatures):
    """Exact e, q^2 and q_l per temperature of a +-J sample (all 2^N states).

    Follows critmc tests/test_glass.py:26-52 (energies as critmc's
    exact/enumeration.py:120-135 ea_energies: E = -sum_b J_b s_i s_j)."""
    n = lattice.n_sites
    bits = np.unpackbits(np.arange(1 << n, dtype=">u4").view(np.uint8).reshape(-1, 4), axis=1,
                         bitorder="big")[:, ::-1][:, :n]  # bit k of the state number is site k
    spins = np.where(bits == 1, 1.0, -1.0)
    i, j = lattice.bonds.T
    energies = -(spins[:, i] * spins[:, j]) @ np.asarray(couplings, dtype=np.float64)
    result = {"e": [], "q2": [], "ql": []}
    for temperature in temperatures:
        weight = np.exp((energies.min() - energies) / temperature)
        weight /= weight.sum()
        two_point = spins.T @ (spins * weight[:, None])  # <s_a s_b>
        result["e"].append(float(weight @ energies) / n)
        result["q2"].append(float(np.square(two_point).sum()) / n ** 2)
        result["ql"].append(float(np.square(two_point[i, j]).mean()))
    return {name: np.array(values) for name, values in result.items()}


def ising_log_g_square6() -> np.ndarray:
    """Exact ln g(E) of the 6x6 Ising torus, levels E = -72 + 4 j (-inf where empty)."""
    import math

    g = [int(v) for v in golden()["ising_dos_square6"]["g"]]
    return np.array([math.log(v) if v > 0 else -np.inf for v in g])


def synthetic_muca(seed: int = 20261204):
    """A seeded bimodal multicanonical record on the q = 10 Potts 8 x 8 levels.

    Energies per site are drawn from two Gaussians (ordered near -1.65,
    disordered near -0.97) inside the window [-1.95, -0.6], with weights
    ln g(E) = 1.40 E + const, so reweighting to beta near 1.40 returns the drawn
    mixture.  Returns (ln_g, level_series, order_series, window, hist) for the
    analysis methods of the multicanonical and Wang-Landau results.
    """
    rng = np.random.default_rng(seed)
    n_sites, n_bonds, levels = 64, 128, 129
    lo, hi = 4, 89  # window [-1.95, -0.6] per site
    n = 40_000
    pick = rng.random(n) < 0.45
    e = np.where(pick, rng.normal(-1.65, 0.06, n), rng.normal(-0.97, 0.09, n))
    idx = np.clip(np.rint(e * n_sites + n_bonds).astype(np.int64), lo, hi)
    energies = np.arange(levels) - float(n_bonds)
    ln_g = 1.40 * energies + 7.0
    order = rng.integers(n_sites ** 2 // 10, n_sites ** 2, n).astype(np.int64)
    hist = np.bincount(idx, minlength=levels).astype(np.int64)
    return ln_g, idx, order, (lo, hi), hist


def fake_advance(call: int, schedule, n_meas: int, n_sites: int, kind: str, n_comp: int = 2) -> dict:
    """Deterministic stand-in for ``Model.advance`` output (call ``call`` of a chain).

    Used to drive critmc's ``Simulation`` (fixture generator) and this
    project's (tests) through the same data, so their host logic -- chunking,
    Wolff-count and Metropolis-step tuning, metadata -- can be compared
    exactly.  Wolff cluster sizes grow with the call index, as for a chain that
    orders while it thermalises.
    """
    rng = np.random.default_rng([7, call])
    sched = np.asarray(schedule).reshape(-1, 2)
    metro = int(sched[np.isin(sched[:, 0], (0, 1)), 1].sum())
    wolff = int(sched[sched[:, 0] == 3, 1].sum())
    aux = np.zeros((n_meas, 4), dtype=np.int64)
    aux[:, 0] = rng.integers(0, metro * n_sites + 1, n_meas)
    aux[:, 1] = wolff * rng.integers(1, min(n_sites, 2 + 3 * call) + 1, n_meas)
    aux[:, 2] = rng.integers(0, n_sites * n_sites, n_meas)
    aux[:, 3] = rng.integers(1, n_sites, n_meas)
    if kind == "on":
        return {"E": rng.normal(-1.0, 0.1, n_meas) * n_sites, "M": rng.normal(size=(n_meas, n_comp)),
                "stiff_c": rng.normal(size=(n_meas, 2)), "stiff_s": rng.normal(size=(n_meas, 2)), "aux": aux}
    e = rng.integers(-2 * n_sites, 2 * n_sites, n_meas)
    return {"E": e, "Eb": e.copy(), "M": rng.integers(-n_sites, n_sites + 1, n_meas), "aux": aux}


# scenarios of the Simulation host-logic comparison: (model, updates, therm, n_chunks, run, chunk)
SIM_SCENARIOS = [
    ("ising", "metropolis+wolff", 100, 10, 700, 300),
    ("ising", "heatbath+3*wolff", 57, 7, 64, 1 << 16),
    ("on", "metropolis+2*overrelax", 90, 9, 50, 20),
    ("ising", "metropolis", 3, 10, 5, 2),
    ("ising", "sw+metropolis", 0, 10, 9, 4),
]


def summarize_series(raw: dict, meta: dict) -> dict:
    """Sums and end values of every stream, and the metadata without wall-clock entries."""
    out = {}
    for k, v in raw.items():
        a = np.asarray(v, dtype=np.float64)
        out[k] = [float(a.sum()), float(a.reshape(len(a), -1)[0, 0]), float(a.reshape(len(a), -1)[-1, -1]),
                  list(a.shape)]
    skip = {"wall_time", "site_updates_per_s", "backend"}
    return {"streams": out, "meta": {k: v for k, v in meta.items() if k not in skip}}
