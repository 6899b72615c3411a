"""Pin the CPU oracle (and the test harness) against critmc's exact results.

The oracle is the bit-exact reference of the GPU kernels; these tests show
that the oracle itself samples the right distributions, by critmc's own
exact layer (fixtures from tests/golden/make_golden.py) and the batch-means
criterion |z| < 4.5 of critmc tests/conftest.py.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import assert_consistent
from exact_helpers import JointDOS, ar1, gamma_error, golden, kaufman_energy

import oracle


@pytest.mark.parametrize("case", golden()["gamma_method_ar1"], ids=lambda c: f"phi{c['phi']}")
def test_gamma_method_matches_critmc(case):
    x = ar1(case["seed"], case["phi"], case["n"])
    m, err, tau = gamma_error(x)
    assert m == pytest.approx(case["value"], rel=1e-12, abs=1e-14)
    assert err == pytest.approx(case["error"], rel=1e-10)
    assert tau == pytest.approx(case["tau_int"], rel=1e-10)


def _ising_state(n, seed):
    return (2 * np.random.default_rng(seed).integers(0, 2, n) - 1).astype(np.int8)


@pytest.mark.parametrize("code", [0, 2])
def test_oracle_byte_ising_matches_enumeration(code):
    jd = JointDOS("ising_dos_square4")
    beta, n = 0.35, 16
    s = _ising_state(n, 1)
    e_b, m, _, _ = oracle.ising_byte_run(s, (4, 4), (3, 4), beta, 0.0, [[code, 1]], 120_000)
    e_b, m = e_b[2000:], m[2000:]
    assert_consistent(e_b, jd.average(beta, lambda e, o: e))
    assert_consistent((m / n) ** 2, jd.average(beta, lambda e, o: (o / n) ** 2))


@pytest.mark.parametrize("code", [0, 2])
def test_oracle_byte_ising_in_a_field(code):
    jd = JointDOS("ising_dos_square4")
    beta, h, n = 0.3, 0.4, 16
    s = _ising_state(n, 2)
    e_b, m, _, _ = oracle.ising_byte_run(s, (4, 4), (5, 6), beta, h, [[code, 1]], 120_000)
    e_b, m = e_b[2000:], m[2000:]
    assert_consistent(e_b - h * m, jd.average(beta, lambda e, o: e - h * o, h=h))
    assert_consistent(m / n, jd.average(beta, lambda e, o: o / n, h=h))


@pytest.mark.parametrize("code", [0, 2])
def test_oracle_potts_matches_enumeration(code):
    jd = JointDOS("potts3_dos_square4x2")
    beta, q, n = 0.8, 3, 8
    s = np.random.default_rng(3).integers(0, q, n).astype(np.int8)
    e, counts, _, _, _ = oracle.potts_run(s, (4, 2), q, (7, 8), beta, [[code, 1]], 150_000)
    e, counts = e[2000:], counts[2000:]
    assert_consistent(e, jd.average(beta, lambda en, o: en))
    rho = counts / n
    m2 = (q * np.sum(rho * rho, axis=1) - 1.0) / (q - 1.0)
    assert_consistent(m2, jd.average(beta, lambda en, o: (o / n ** 2 - 1.0) / (q - 1.0)))


@pytest.mark.parametrize("code", [0, 2])
def test_oracle_msc_matches_kaufman(code):
    """The multi-spin-coded stream samples the 64x4 torus (Kaufman's exact energy)."""
    beta = 0.4
    s = _ising_state(256, 4)
    e_b, _, _, _ = oracle.ising_msc_run(s, (64, 4), (9, 10), beta, 0.0, [[code, 1]], 40_000)
    assert_consistent(e_b[1000:] / 256.0, kaufman_energy(beta, 64, 4))


@pytest.mark.parametrize("n", [2, 3])
@pytest.mark.parametrize("sched", [[[2, 1]], [[0, 1], [5, 3]]], ids=["heatbath", "metropolis+3*overrelax"])
def test_oracle_on_ring_matches_transfer_operator(n, sched):
    """critmc tests/test_kernels.py:95-109: 8-site O(n) ring against chains.on_ring_*."""
    ref = golden()["on_ring"][f"n{n}_N8_b1.1"]
    rng = np.random.default_rng(n)
    s = rng.standard_normal((8, n))
    s = (s / np.linalg.norm(s, axis=1, keepdims=True)).astype(np.float32)
    e, _, _, _, _ = oracle.on_run(s, (8,), n, (n, 5), 1.1, 1.0, sched, 100_000)
    e = e[2000:]
    assert_consistent(e / 8.0, ref["energy"])
    c_mc = 1.1 ** 2 * e.var() / 8
    assert c_mc == pytest.approx(ref["specific_heat"], rel=0.06)


@pytest.mark.parametrize("n", [2, 3])
@pytest.mark.parametrize("algo,reps", [(3, 3), (4, 1)], ids=["3*wolff", "sw"])
def test_oracle_on_cluster_ring_matches_transfer_operator(n, algo, reps):
    """Embedded-Ising cluster updates alone (critmc kernels/on.py:265-345) on the
    8-site O(n) ring against chains.on_ring_*; spins renormalised per measurement."""
    from critmc_b200.layout import cb_pack, cb_unpack

    ref = golden()["on_ring"][f"n{n}_N8_b1.1"]
    rng = np.random.default_rng(10 + n)
    s = rng.standard_normal((8, n))
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    comps = np.ascontiguousarray(np.stack([cb_pack(s[:, k], (8,)) for k in range(n)]).astype(np.float32))
    comps = comps.reshape(n, -1)
    n_meas, sweep, e = 40_000, 0, []
    for _ in range(n_meas):
        for _ in range(reps):
            oracle.on_cluster_update(comps, (8,), (n, 17), 1.1, algo, sweep)
            sweep += 1
        comps /= np.sqrt((comps.astype(np.float64) ** 2).sum(axis=0)).astype(np.float32)
        v = np.stack([cb_unpack(comps[k], (8,)) for k in range(n)], axis=1).astype(np.float64)
        e.append(-np.sum(v * np.roll(v, -1, axis=0)))
    e = np.array(e[1000:])
    assert_consistent(e / 8.0, ref["energy"])
    assert 1.1 ** 2 * e.var() / 8 == pytest.approx(ref["specific_heat"], rel=0.08)


def test_ea_enumeration_helper_matches_critmc():
    """The test-side EA enumeration reproduces critmc's ea_energies fixture."""
    from critmc_b200 import square

    g = golden()["ea_square4"]
    lat = square(4)
    n = lat.n_sites
    states = np.arange(64)
    spins = (2 * ((states[:, None] >> np.arange(n)) & 1) - 1).astype(np.float64)
    b = lat.bonds
    e = -(spins[:, b[:, 0]] * spins[:, b[:, 1]]) @ np.asarray(g["couplings"])
    np.testing.assert_allclose(e, g["energies_first_64"])


def test_oracle_parallel_tempering_matches_enumeration():
    """critmc tests/test_glass.py:26-52 for a +-J 4x4 sample, on the CPU oracle."""
    from exact_helpers import ea_exact

    from critmc_b200 import square
    from critmc_b200.glass import geometric_temperatures

    lat = square(4)
    J = np.asarray(golden()["ea_square4"]["couplings"])
    temps = geometric_temperatures(0.4, 2.5, 8)[::-1].copy()  # hot -> cold
    betas = 1.0 / temps
    m, n = 8, 16
    rng = np.random.default_rng(5)
    spins = (2 * rng.integers(0, 2, size=(2, m, n)) - 1).astype(np.int8)
    perm = np.tile(np.arange(m, dtype=np.int32), (2, 1))
    labels = np.zeros((2, m), dtype=np.int32)
    from critmc_b200 import _lib

    table = np.zeros((m - 1, 2048), dtype=np.uint32)
    _lib.call("critmc_pt_swap_table", m, np.ascontiguousarray(betas).ctypes.data, 2048, table.ctypes.data)
    acc, sa, st, lh, tr = oracle.ea_pt_run(spins, J, (4, 4), np.array([[1, 2], [3, 4]]), betas, table,
                                           perm, labels, n_steps=(1 << 14) - 1, n_bins=14)
    eq = acc[-1] / acc[-1][:, 6:7]
    ex = ea_exact(lat, J, temps)
    np.testing.assert_allclose(eq[:, 0], ex["e"], atol=0.01)
    np.testing.assert_allclose(eq[:, 3], ex["q2"], atol=0.02)
    np.testing.assert_allclose(eq[:, 1], ex["ql"], atol=0.02)
    assert np.all(sa / st > 0.3)
    assert tr.sum() > 50
