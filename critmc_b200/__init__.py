"""critmc_b200: critmc's data-parallel sampling path, rebuilt for the NVIDIA B200.

Checkerboard Metropolis and heat-bath sweeps for the Ising model (with
field), the q-state Potts model, the O(n) models (XY, Heisenberg, with
over-relaxation) and Edwards-Anderson +-J spin glasses with parallel
tempering, as hand-written sm_100a CUDA kernels behind a C ABI
(``include/critmc_b200.h``).  The Python layer keeps critmc's
``Simulation(model, beta, updates=..., seed=...)`` / ``thermalize`` / ``run``
API and its update-schedule strings.
"""

from .lattice import Lattice, chain, cubic, hypercubic, make_lattice, square, triangular
from .models import ON, XY, Heisenberg, Ising, Model, Potts, build_model, derive
from .rng import make_rng, philox_key, spawn_rngs
from .sim import Simulation, TimeSeries, parse_updates

__version__ = "1.0.0"

__all__ = [
    "Lattice",
    "chain",
    "square",
    "cubic",
    "triangular",
    "hypercubic",
    "make_lattice",
    "Model",
    "Ising",
    "Potts",
    "ON",
    "XY",
    "Heisenberg",
    "build_model",
    "derive",
    "Simulation",
    "TimeSeries",
    "parse_updates",
    "make_rng",
    "spawn_rngs",
    "philox_key",
    "__version__",
]
