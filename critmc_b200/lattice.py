"""Periodic lattices with critmc's site numbering.

Same tables as critmc ``src/critmc/lattice.py:26-221``, so configurations move
between the two packages unchanged:

- sites are numbered with the first coordinate fastest,
  ``i = x0 + L0 (x1 + L1 x2)`` (critmc lattice.py:118-127);
- the neighbour table ``nbr`` (N, z) has its columns in opposite pairs, column
  ``2a`` the neighbour along +e_a and ``2a+1`` along -e_a;
- the bonds are (site, forward neighbour) for axis 0, then axis 1, ..., each in
  site order, with ``bond_axis`` the axis of each;
- ``coords`` are the integer coordinates, ``positions`` the Cartesian ones.

A hypercubic lattice with every extent even is bipartite (``sublattice`` is the
parity of the coordinate sum), which the checkerboard sweeps require.
"""

from __future__ import annotations

from dataclasses import dataclass
from math import prod

import numpy as np

__all__ = ["Lattice", "hypercubic", "chain", "square", "cubic", "triangular", "make_lattice"]


@dataclass(frozen=True, eq=False)
class Lattice:
    name: str
    shape: tuple[int, ...]
    nbr: np.ndarray
    bonds: np.ndarray
    bond_axis: np.ndarray
    positions: np.ndarray
    coords: np.ndarray
    primitive: np.ndarray
    sublattice: np.ndarray | None

    @property
    def n_sites(self) -> int:
        return len(self.nbr)

    @property
    def z(self) -> int:
        return self.nbr.shape[1]

    @property
    def dim(self) -> int:
        return len(self.shape)

    @property
    def n_bonds(self) -> int:
        return len(self.bonds)

    @property
    def L(self) -> int:
        return self.shape[0]

    @property
    def bipartite(self) -> bool:
        return self.sublattice is not None

    @property
    def hypercubic(self) -> bool:
        return self.name in ("chain", "square", "cubic") or self.name.startswith("hypercubic")

    def site(self, *x: int) -> int:
        """Index of the site at coordinates ``x`` (taken modulo the extents)."""
        if len(x) != len(self.shape):
            raise ValueError(f"a site of this {len(self.shape)}-dimensional lattice needs that many coordinates, "
                             f"got {len(x)}")
        return int(np.ravel_multi_index(tuple(int(c) for c in x), self.shape, mode="wrap", order="F"))

    def reciprocal(self) -> np.ndarray:
        """Rows b_j with a_i . b_j = 2 pi delta_ij for the primitive rows a_i."""
        return 2.0 * np.pi * np.linalg.inv(self.primitive).T

    def kmin(self, axis: int = 0) -> np.ndarray:
        """The smallest wave vector along ``axis`` that fits the torus."""
        return self.reciprocal()[axis] / self.shape[axis]

    def __repr__(self) -> str:
        return "Lattice({}, {}, N={}, z={})".format(self.name, "x".join(map(str, self.shape)), self.n_sites, self.z)


def _extents(shape) -> tuple[int, ...]:
    ext = tuple(map(int, shape))
    if len(ext) == 0:
        raise ValueError("a lattice has at least one extent")
    if any(e < 2 for e in ext):
        raise ValueError(f"every linear extent must be >= 2, got {ext}")
    return ext


def _coordinates(shape: tuple[int, ...]) -> np.ndarray:
    """(N, d) coordinates of the sites, first coordinate fastest."""
    return np.stack(np.unravel_index(np.arange(prod(shape)), shape, order="F"), axis=1).astype(np.int64)


def _shifted(coords: np.ndarray, shape: tuple[int, ...], step: np.ndarray) -> np.ndarray:
    """Index of the site at ``coords + step`` on the torus."""
    return np.ravel_multi_index(tuple((coords + step).T), shape, mode="wrap", order="F").astype(np.int64)


def _tables(coords, shape, steps):
    """Neighbour columns (+step, -step per direction), bonds and their axes."""
    n = len(coords)
    nbr = np.stack([_shifted(coords, shape, sign * np.asarray(step))
                    for step in steps for sign in (1, -1)], axis=1)
    here = np.arange(n, dtype=np.int64)
    bonds = np.concatenate([np.column_stack((here, nbr[:, 2 * a])) for a in range(len(steps))])
    bond_axis = np.arange(len(steps), dtype=np.int64).repeat(n)
    return nbr, bonds, bond_axis


def hypercubic(shape, name: str | None = None) -> Lattice:
    """Periodic hypercubic lattice of the given extents; first coordinate fastest."""
    ext = _extents(shape)
    d = len(ext)
    coords = _coordinates(ext)
    nbr, bonds, bond_axis = _tables(coords, ext, list(np.eye(d, dtype=np.int64)))
    parity = (coords.sum(axis=1) % 2).astype(np.int8) if all(e % 2 == 0 for e in ext) else None
    label = name or {1: "chain", 2: "square", 3: "cubic"}.get(d, f"hypercubic{d}d")
    return Lattice(label, ext, nbr, bonds, bond_axis, coords.astype(np.float64), coords, np.eye(d), parity)


def chain(L: int) -> Lattice:
    return hypercubic((L,), name="chain")


def square(L: int, M: int | None = None) -> Lattice:
    return hypercubic((L, M or L), name="square")


def cubic(L: int) -> Lattice:
    return hypercubic((L,) * 3, name="cubic")


_TRIANGLE = np.array([[1.0, 0.0], [0.5, 0.5 * np.sqrt(3.0)]])


def triangular(L: int, M: int | None = None) -> Lattice:
    """Triangular torus (coordination 6, directions (1,0), (0,1), (1,-1) in the
    primitive basis).  Not bipartite: the checkerboard samplers refuse it
    (critmc lattice.py:173-205 builds the same geometry)."""
    ext = _extents((L, M or L))
    coords = _coordinates(ext)
    nbr, bonds, bond_axis = _tables(coords, ext, [np.array(s) for s in ((1, 0), (0, 1), (1, -1))])
    return Lattice("triangular", ext, nbr, bonds, bond_axis, coords @ _TRIANGLE, coords, _TRIANGLE.copy(), None)


_BUILDERS = {"chain": chain, "square": square, "cubic": cubic, "triangular": triangular}


def make_lattice(name: str, L: int) -> Lattice:
    """The lattice of a model spec (``"chain"``, ``"square"``, ``"cubic"``, ``"triangular"``)."""
    if name not in _BUILDERS:
        raise ValueError(f"unknown lattice {name!r}; the lattices are {sorted(_BUILDERS)}")
    return _BUILDERS[name](L)
