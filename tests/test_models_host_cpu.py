"""Model host methods against critmc's own (critmc models.py:32-351, fixture):
seeded initial states (same generator draws), energies, metadata and the
derived per-site observables; and build_model from a spec."""

from __future__ import annotations

import numpy as np
import pytest
from exact_helpers import golden

from critmc_b200 import ON, Ising, Potts, build_model, chain, cubic, derive, make_rng, square


def _models():
    return {"ising": Ising(square(6), h=0.25), "potts": Potts(cubic(4), 5), "on": ON(chain(8), 3)}


@pytest.mark.parametrize("name", ["ising", "potts", "on"])
def test_model_host_methods_match_critmc(name):
    ref = golden()["model_host"][name]
    mdl = _models()[name]
    s0 = mdl.initial_state("random", make_rng(3, "start"))
    np.testing.assert_array_equal(np.asarray(s0, dtype=np.float64).ravel(), ref["random"])
    s1 = mdl.initial_state("ordered", make_rng(3))
    np.testing.assert_array_equal(np.asarray(s1, dtype=np.float64).ravel(), ref["ordered"])
    assert mdl.energy(s0) == pytest.approx(ref["energy_random"], rel=1e-12, abs=1e-12)
    assert mdl.meta() == ref["meta"] and mdl.spec() == ref["spec"]
    assert build_model(ref["spec"]).meta() == ref["meta"]
    with pytest.raises(ValueError):
        mdl.initial_state("sideways", make_rng(1))


def test_derived_observables_match_critmc():
    rng = np.random.default_rng(99)
    raws = {"ising": ({"E": rng.integers(-72, 72, 20).astype(float), "M": rng.integers(-36, 37, 20)},
                      {"model": "ising", "N": 36}),
            "potts": ({"E": rng.integers(-192, 0, 20).astype(float), "counts": rng.multinomial(64, [0.2] * 5, 20)},
                      {"model": "potts", "N": 64, "q": 5}),
            "on": ({"E": rng.normal(size=20), "M": rng.normal(size=(20, 3)) * 3}, {"model": "on", "N": 8})}
    for name, (raw, meta) in raws.items():
        ref = golden()["model_host"][name]["derive"]
        got = derive(raw, meta)
        assert set(got) == set(ref), name
        for k, v in ref.items():
            np.testing.assert_allclose(got[k], v, rtol=1e-13, atol=1e-15, err_msg=f"{name}.{k}")
    with pytest.raises(ValueError):
        derive({"E": np.zeros(2)}, {"model": "clock", "N": 4})


def test_edwards_anderson_samples_match_critmc():
    """+-J couplings for a seed, the geometric temperatures and the sample energy as
    critmc's (critmc glass.py:45-95, fixture)."""
    from critmc_b200.glass import EdwardsAnderson, geometric_temperatures

    ref = golden()["ea_samples"]
    for sd in (1, 2):
        sample = EdwardsAnderson(cubic(4), disorder="bimodal", seed=sd)
        np.testing.assert_array_equal(sample.couplings, ref["cubic4"][str(sd)]["couplings"])
        state = np.where(np.random.default_rng(sd).random(64) < 0.5, -1, 1)
        assert sample.energy(state) == ref["cubic4"][str(sd)]["energy"]
    np.testing.assert_allclose(geometric_temperatures(0.5, 2.0, 32), ref["temperatures"], rtol=1e-15)
    with pytest.raises(ValueError):
        EdwardsAnderson(cubic(4), disorder="gaussian", seed=1)
    with pytest.raises(ValueError):
        EdwardsAnderson(cubic(4), couplings=np.ones(5))


def test_edwards_anderson_default_is_critmcs_gaussian_and_refused():
    """critmc's EdwardsAnderson defaults to Gaussian couplings (critmc glass.py:52); the
    +-J kernel refuses that default and names the disorder it runs, instead of
    silently building a different model for the same call."""
    from critmc_b200.glass import EdwardsAnderson

    with pytest.raises(ValueError, match='disorder="bimodal"'):
        EdwardsAnderson(cubic(4), seed=1)
    assert EdwardsAnderson(cubic(4), disorder="bimodal", seed=1).disorder == "bimodal"
