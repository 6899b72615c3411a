"""Periodic lattices with critmc's site numbering.

Same contract as critmc ``src/critmc/lattice.py:26-221``: a lattice carries a
neighbour table ``nbr`` (N, z) whose columns come in opposite pairs
(``2a`` = +e_a, ``2a+1`` = -e_a), a bond list built from the forward columns,
``bond_axis``, integer ``coords`` and Cartesian ``positions``.  Sites are
numbered with the first coordinate fastest, ``i = x0 + L0 (x1 + L1 x2)``
(critmc lattice.py:118-127), so configurations move between the two packages
unchanged.

The GPU samplers only need the extents: a hypercubic lattice with every
extent even is bipartite, which is what the checkerboard sweeps require
(critmc lattice.py:140-141 defines ``sublattice`` under the same condition).
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
        return int(self.nbr.shape[0])

    @property
    def z(self) -> int:
        return int(self.nbr.shape[1])

    @property
    def dim(self) -> int:
        return len(self.shape)

    @property
    def n_bonds(self) -> int:
        return int(self.bonds.shape[0])

    @property
    def L(self) -> int:
        return int(self.shape[0])

    @property
    def bipartite(self) -> bool:
        return self.sublattice is not None

    @property
    def hypercubic(self) -> bool:
        return self.name in ("chain", "square", "cubic") or self.name.startswith("hypercubic")

    def site(self, *x: int) -> int:
        if len(x) != self.dim:
            raise ValueError(f"expected {self.dim} coordinates, got {len(x)}")
        idx = 0
        for c, n in zip(reversed(x), reversed(self.shape)):
            idx = idx * n + int(c) % n
        return idx

    def reciprocal(self) -> np.ndarray:
        return 2.0 * np.pi * np.linalg.inv(self.primitive).T

    def kmin(self, axis: int = 0) -> np.ndarray:
        return self.reciprocal()[axis] / self.shape[axis]

    def __repr__(self) -> str:
        return f"Lattice({self.name}, {'x'.join(map(str, self.shape))}, N={self.n_sites}, z={self.z})"


def _extents(shape) -> tuple[int, ...]:
    out = tuple(int(n) for n in shape)
    if not out:
        raise ValueError("lattice needs at least one dimension")
    if min(out) < 2:
        raise ValueError(f"every linear extent must be >= 2, got {out}")
    return out


def _coords(shape: tuple[int, ...]) -> np.ndarray:
    n = prod(shape)
    idx = np.arange(n, dtype=np.int64)
    cols = []
    for extent in shape:
        cols.append(idx % extent)
        idx = idx // extent
    return np.stack(cols, axis=1)


def _index(coords: np.ndarray, shape: tuple[int, ...]) -> np.ndarray:
    idx = np.zeros(coords.shape[0], dtype=np.int64)
    for a in reversed(range(len(shape))):
        idx = idx * shape[a] + coords[:, a]
    return idx


def hypercubic(shape, name: str | None = None) -> Lattice:
    """Periodic hypercubic lattice; first coordinate fastest."""
    shape = _extents(shape)
    d = len(shape)
    coords = _coords(shape)
    n = coords.shape[0]
    nbr = np.empty((n, 2 * d), dtype=np.int64)
    for a in range(d):
        for col, step in ((2 * a, 1), (2 * a + 1, -1)):
            moved = coords.copy()
            moved[:, a] = (moved[:, a] + step) % shape[a]
            nbr[:, col] = _index(moved, shape)
    sites = np.arange(n, dtype=np.int64)
    bonds = np.concatenate([np.stack([sites, nbr[:, 2 * a]], axis=1) for a in range(d)])
    bond_axis = np.repeat(np.arange(d, dtype=np.int64), n)
    sublattice = None
    if all(e % 2 == 0 for e in shape):
        sublattice = (coords.sum(axis=1) % 2).astype(np.int8)
    if name is None:
        name = {1: "chain", 2: "square", 3: "cubic"}.get(d, f"hypercubic{d}d")
    return Lattice(name, shape, nbr, bonds, bond_axis, coords.astype(np.float64), coords,
                   np.eye(d), sublattice)


def chain(L: int) -> Lattice:
    return hypercubic((L,), name="chain")


def square(L: int, M: int | None = None) -> Lattice:
    return hypercubic((L, L if M is None else M), name="square")


def cubic(L: int) -> Lattice:
    return hypercubic((L, L, L), name="cubic")


def triangular(L: int, M: int | None = None) -> Lattice:
    """Triangular torus (coordination 6).  Not bipartite: the checkerboard
    samplers refuse it (critmc lattice.py:173-205 builds the same geometry)."""
    shape = _extents((L, L if M is None else M))
    coords = _coords(shape)
    n = coords.shape[0]
    nbr = np.empty((n, 6), dtype=np.int64)
    for a, (dx, dy) in enumerate(((1, 0), (0, 1), (1, -1))):
        for col, sgn in ((2 * a, 1), (2 * a + 1, -1)):
            moved = np.stack([(coords[:, 0] + sgn * dx) % shape[0], (coords[:, 1] + sgn * dy) % shape[1]], 1)
            nbr[:, col] = _index(moved, shape)
    sites = np.arange(n, dtype=np.int64)
    bonds = np.concatenate([np.stack([sites, nbr[:, 2 * a]], axis=1) for a in range(3)])
    bond_axis = np.repeat(np.arange(3, dtype=np.int64), n)
    primitive = np.array([[1.0, 0.0], [0.5, np.sqrt(3.0) / 2.0]])
    return Lattice("triangular", shape, nbr, bonds, bond_axis, coords @ primitive, coords,
                   primitive, None)


_BUILDERS = {"chain": chain, "square": square, "cubic": cubic, "triangular": triangular}


def make_lattice(name: str, L: int) -> Lattice:
    try:
        return _BUILDERS[name](L)
    except KeyError:
        raise ValueError(f"unknown lattice {name!r}; choose from {sorted(_BUILDERS)}") from None
