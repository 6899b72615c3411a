"""The no-allocation variant of the multi-spin-coded Ising entry point.

critmc_ising_msc_run_noalloc serves callers that cannot call cudaMalloc where
they run the sampler (a plugin whose framework owns the device allocator, code
that must not stall the device with an allocation, hosts that forbid
allocation after start-up): it keeps its accumulators in a 1 MiB array built
into the library instead of a caller buffer.  This file is collected last on
purpose; the test also passes alone in a fresh process.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from critmc_b200 import Ising, _lib, square
from critmc_b200.lattice import hypercubic
from critmc_b200.device import empty_bytes, ptr, stream_handle, to_dev, to_host
from critmc_b200.layout import msc_pack

pytestmark = pytest.mark.gpu


def _state(shape, n_chains, seed):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    return [(2 * rng.integers(0, 2, n) - 1).astype(np.int8) for _ in range(n_chains)]


def _compare_two_calls(cuda, shape, n_chains, n_meas, betas, sched, seed):
    """Run the allocating entry point and the no-allocation one side by side on
    the same chains, twice in a row, and require identical results."""
    dim = len(shape)
    lx, ly = shape[0], shape[1]
    lz = shape[2] if dim == 3 else 1
    lat = square(lx, ly) if dim == 2 else hypercubic((lx, ly, lz))
    model = Ising(lat)
    states = _state(shape, n_chains, seed)
    keys = np.random.default_rng(seed + 1).integers(0, 2**32, (n_chains, 2), dtype=np.uint64).astype(np.uint32)
    tables = np.ascontiguousarray(np.stack([model.tables(b)[0] for b in betas]))
    sched = np.asarray(sched, dtype=np.int64)
    words = np.stack([msc_pack(s, shape) for s in states])
    run0 = np.array([[model.bond_energy(s), int(s.astype(np.int64).sum())] for s in states], np.int64)

    def buffers():
        return (to_dev(words, cuda), torch.from_numpy(run0.copy()).to(cuda),
                torch.empty((n_chains, n_meas), dtype=torch.int64, device=cuda),
                torch.empty((n_chains, n_meas), dtype=torch.int64, device=cuda),
                torch.empty((n_chains, n_meas, 4), dtype=torch.int64, device=cuda))

    ref_w, ref_run, ref_e, ref_m, ref_aux = buffers()
    new_w, new_run, new_e, new_m, new_aux = buffers()
    scratch = empty_bytes(_lib.lib().critmc_ising_msc_scratch_bytes(n_chains, n_meas), cuda)
    st = stream_handle(cuda)
    per_meas = int(sched[:, 1].sum())
    for call in range(2):  # the second call starts from the state the first one left
        sweep0 = call * n_meas * per_meas
        _lib.call("critmc_ising_msc_run", ptr(ref_w), dim, lx, ly, lz, n_chains, keys.ctypes.data,
                  tables.ctypes.data, len(betas), sweep0, sched.ctypes.data, len(sched), n_meas, ptr(ref_run),
                  ptr(ref_e), ptr(ref_m), ptr(ref_aux), ptr(scratch), 3, 8, st)
        _lib.call("critmc_ising_msc_run_noalloc", ptr(new_w), dim, lx, ly, lz, n_chains,
                  keys.ctypes.data, tables.ctypes.data, len(betas), sweep0, sched.ctypes.data, len(sched),
                  n_meas, ptr(new_run), ptr(new_e), ptr(new_m), ptr(new_aux), 8, st)
        torch.cuda.synchronize(cuda)
        # integer series and spins: the tolerance of these kernels is exact equality
        np.testing.assert_array_equal(to_host(new_e), to_host(ref_e))
        np.testing.assert_array_equal(to_host(new_m), to_host(ref_m))
        np.testing.assert_array_equal(to_host(new_aux), to_host(ref_aux))
        np.testing.assert_array_equal(to_host(new_run), to_host(ref_run))
        np.testing.assert_array_equal(to_host(new_w), to_host(ref_w))


@pytest.mark.parametrize("shape,n_chains,betas", [
    ((256, 64), 4, (0.42, 0.46)),      # 2D, two chain groups
    ((64, 8, 6), 4, (0.21, 0.23)),     # 3D (six neighbours), two chain groups
    ((128, 16, 4), 3, (0.2216,)),      # 3D, one group
])
def test_noalloc_matches_the_allocating_entry_point_on_two_calls(cuda, shape, n_chains, betas):
    _compare_two_calls(cuda, shape, n_chains, 9, betas, [[0, 1], [2, 1]], 3)


def test_noalloc_at_exactly_its_scratch_limit(cuda):
    """n_chains * n_meas = 43,690 fills the 1 MiB array to its last byte: the
    clearing of the accumulators and the indexing of the last measurement
    meet the end of the array there."""
    lib = _lib.lib()
    n_chains, n_meas = 10, 4369
    assert lib.critmc_ising_msc_scratch_bytes(n_chains, n_meas) == lib.critmc_ising_msc_noalloc_max_scratch_bytes()
    _compare_two_calls(cuda, (64, 4), n_chains, n_meas, (0.40, 0.48), [[0, 1]], 11)


def test_noalloc_rejects_calls_beyond_its_scratch(cuda):
    lib = _lib.lib()
    cap = lib.critmc_ising_msc_noalloc_max_scratch_bytes()
    assert cap == 1 << 20
    n_chains, n_meas = 2, 30_000  # 16 + 2 * 30000 * 24 bytes > 1 MiB
    assert lib.critmc_ising_msc_scratch_bytes(n_chains, n_meas) > cap
    keys = np.zeros((n_chains, 2), np.uint32)
    tables = np.ascontiguousarray(np.stack([Ising(square(64)).tables(0.4)[0]]))
    sched = np.array([[0, 1]], np.int64)
    dummy = torch.empty(16, dtype=torch.int64, device=cuda)
    st = lib.critmc_ising_msc_run_noalloc(ptr(dummy), 2, 64, 64, 1, n_chains, keys.ctypes.data,
                                          tables.ctypes.data, 1, 0, sched.ctypes.data, 1, n_meas,
                                          ptr(dummy), ptr(dummy), ptr(dummy), ptr(dummy), 8,
                                          stream_handle(cuda))
    assert st == -1
    assert "1 MiB" in _lib.last_error()
