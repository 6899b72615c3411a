"""Site numbering, neighbour and bond tables, and keyed random streams against
critmc's own (critmc lattice.py:118-213, rng.py:28-66; fixture): both are part
of the drop-in contract (same sites, same seeds give the same streams)."""

from __future__ import annotations

import numpy as np
import pytest
from exact_helpers import golden

from critmc_b200 import chain, cubic, hypercubic, make_lattice, make_rng, spawn_rngs, square, triangular


def _lattices():
    return {"chain6": chain(6), "square4x3": square(4, 3), "cubic3": cubic(3),
            "hyper2x2x2x2": hypercubic((2, 2, 2, 2)), "triangular4": triangular(4),
            "square_named": make_lattice("square", 5)}


@pytest.mark.parametrize("name", ["chain6", "square4x3", "cubic3", "hyper2x2x2x2", "triangular4", "square_named"])
def test_lattice_tables_match_critmc(name):
    ref = golden()["lattices"][name]
    lat = _lattices()[name]
    assert lat.name == ref["name"] and list(lat.shape) == ref["shape"] and lat.z == ref["z"]
    for key in ("nbr", "bonds", "bond_axis", "coords"):
        np.testing.assert_array_equal(getattr(lat, key), ref[key], err_msg=key)
    np.testing.assert_allclose(lat.positions, ref["positions"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(lat.primitive, ref["primitive"], rtol=0, atol=1e-15)
    if ref["sublattice"] is None:
        assert lat.sublattice is None and not lat.bipartite
    else:
        np.testing.assert_array_equal(lat.sublattice, ref["sublattice"])
    assert lat.site(*([1] * lat.dim)) == ref["site_ones"]
    np.testing.assert_allclose(lat.kmin(0), ref["kmin"], rtol=1e-14)


def test_bad_lattices_and_coordinates():
    with pytest.raises(ValueError):
        make_lattice("honeycomb", 4)
    with pytest.raises(ValueError):
        square(4).site(1)
    with pytest.raises(ValueError):
        hypercubic(())


def test_keyed_streams_match_critmc():
    ref = golden()["rng_streams"]
    cases = {"int": (5,), "int_keys": (5, "ising", 64, 2), "str_key": (123, "walker", 7), "tuple_key": (9, (1, 2)),
             "bool_key": (4, True, False), "float_key": (4, 0.5), "seedseq": (np.random.SeedSequence(77),),
             "seedseq_keys": (np.random.SeedSequence(77), 3)}
    for label, args in cases.items():
        assert make_rng(*args).integers(0, 2**32, size=4).tolist() == ref[label], label
    assert [g.integers(0, 2**32, size=2).tolist() for g in spawn_rngs(8, 3, "x")] == ref["spawn"]
    g = np.random.default_rng(1)
    assert make_rng(g) is g
    with pytest.raises(ValueError):
        make_rng(g, "key")
    with pytest.raises(ValueError):
        make_rng(1, -3)
