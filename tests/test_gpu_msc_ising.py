"""Multi-spin-coded Ising kernels against the CPU replay: bit-identical spins and series."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from critmc_b200 import Ising, hypercubic, _lib
from critmc_b200.device import empty_bytes, ptr, stream_handle, to_dev, to_host
from critmc_b200.layout import msc_pack, msc_unpack
from critmc_b200.models import _IsingMscChain

pytestmark = pytest.mark.gpu

CASES = [
    # shape, schedule, beta, h
    ((64, 2), [[0, 1]], 0.4406868, 0.0),
    ((64, 64), [[0, 1]], 0.4406868, 0.0),
    ((128, 6), [[2, 1]], 0.4406868, 0.0),
    ((256, 8), [[0, 2], [2, 1]], 0.3, 0.0),
    ((64, 4), [[0, 1]], 1.2, 0.0),
    ((64, 4), [[0, 1]], 0.05, 0.0),
    ((64, 6), [[0, 1]], 0.4, 0.35),
    ((64, 6), [[2, 1]], 0.4, -0.5),
    ((64, 4, 4), [[0, 1]], 0.2216546, 0.0),
    ((64, 2, 6), [[2, 1], [0, 1]], 0.3, 0.2),
]


def _run_gpu(cuda, shape, sched, beta, h, s0, key, n_meas, mode, k_inline, chunks):
    model = Ising(hypercubic(shape), h)
    chain = _IsingMscChain(model, s0, key, cuda)
    chain.mode, chain.k_inline = mode, k_inline
    running = model.begin(s0)
    parts = []
    for k in chunks:
        parts.append(model.advance(chain, running, beta, np.array(sched), k))
    raw = {key_: np.concatenate([p[key_] for p in parts]) for key_ in parts[0]}
    return raw, chain.fetch(), running


@pytest.mark.parametrize("shape,sched,beta,h", CASES)
@pytest.mark.parametrize("mode,k_inline", [(1, 8), (3, 4)])
def test_msc_bit_identical_to_replay(cuda, shape, sched, beta, h, mode, k_inline):
    rng = np.random.default_rng(hash((shape, beta, h)) % 2**32)
    n = int(np.prod(shape))
    s0 = (2 * rng.integers(0, 2, n) - 1).astype(np.int8)
    key = rng.integers(0, 2**32, 2, dtype=np.uint64).astype(np.uint32)
    n_meas = 23
    raw, s_gpu, running = _run_gpu(cuda, shape, sched, beta, h, s0, key, n_meas, mode, k_inline,
                                   chunks=[9, 14])
    s_ref = s0.copy()
    e, m, aux, run = oracle.ising_msc_run(s_ref, shape, key, beta, h, sched, n_meas)
    np.testing.assert_array_equal(s_gpu, s_ref)
    np.testing.assert_array_equal(raw["Eb"], e)
    np.testing.assert_array_equal(raw["M"], m)
    np.testing.assert_array_equal(raw["aux"], aux)
    assert running["e_b"] == run[0] and running["m"] == run[1]


def test_msc_batched_chains_match_single_chain_replays(cuda):
    """Many chains in one launch give each chain's own replay (independent of batching)."""
    shape, beta, n_chains, n_meas = (128, 8), 0.4406868, 5, 11
    lx, ly = shape
    model = Ising(hypercubic(shape))
    rng = np.random.default_rng(11)
    states = [(2 * rng.integers(0, 2, lx * ly) - 1).astype(np.int8) for _ in range(n_chains)]
    keys = rng.integers(0, 2**32, (n_chains, 2), dtype=np.uint64).astype(np.uint32)
    words = to_dev(np.stack([msc_pack(s, shape) for s in states]), cuda)
    tables, _ = model.tables(beta)
    running = torch.tensor([[model.bond_energy(s), int(s.sum())] for s in states],
                           dtype=torch.int64, device=cuda)
    e = torch.empty((n_chains, n_meas), dtype=torch.int64, device=cuda)
    m = torch.empty_like(e)
    aux = torch.empty((n_chains, n_meas, 4), dtype=torch.int64, device=cuda)
    scratch = empty_bytes(_lib.lib().critmc_ising_msc_scratch_bytes(n_chains, n_meas), cuda)
    sched = np.array([[0, 1]], dtype=np.int64)
    _lib.call("critmc_ising_msc_run", ptr(words), 2, lx, ly, 1, n_chains, keys.ctypes.data,
              tables.ctypes.data, 1, 17, sched.ctypes.data, 1, n_meas, ptr(running), ptr(e), ptr(m),
              ptr(aux), ptr(scratch), 3, 8, stream_handle(cuda))
    torch.cuda.synchronize()
    w_host = to_host(words, np.uint32)
    for c in range(n_chains):
        s_ref = states[c].copy()
        er, mr, auxr, _ = oracle.ising_msc_run(s_ref, shape, keys[c], beta, 0.0, sched, n_meas,
                                               sweep0=17)
        np.testing.assert_array_equal(msc_unpack(w_host[c], shape), s_ref)
        np.testing.assert_array_equal(to_host(e)[c], er)
        np.testing.assert_array_equal(to_host(m)[c], mr)
        np.testing.assert_array_equal(to_host(aux)[c], auxr)


def test_msc_measure_matches_host(cuda):
    rng = np.random.default_rng(2)
    for shape in [(64, 64), (128, 4, 6)]:
        lat = hypercubic(shape)
        s = (2 * rng.integers(0, 2, lat.n_sites) - 1).astype(np.int8)
        words = to_dev(msc_pack(s, shape)[None], cuda)
        out = torch.empty((1, 2), dtype=torch.int64, device=cuda)
        dims = tuple(shape) + (1,) * (3 - len(shape))
        _lib.call("critmc_ising_msc_measure", ptr(words), len(shape), *dims, 1, ptr(out),
                  stream_handle(cuda))
        e_b, mm = to_host(out)[0]
        assert e_b == Ising(lat).bond_energy(s)
        assert mm == int(s.astype(np.int64).sum())


@pytest.mark.parametrize("shape,sched,beta", [
    ((128, 8), [[0, 1], [2, 1]], 0.4406868),
    ((64, 4, 6), [[0, 1]], 0.2216546),
])
@pytest.mark.parametrize("mode,k_inline", [(1, 8), (3, 4)])
def test_msc_philox7_planes_replay(cuda, shape, sched, beta, mode, k_inline):
    """The optional Philox4x32-7 acceptance planes (mode bit 12) follow the oracle with
    rounds = 7, and are a different stream from the default Philox4x32-10."""
    philox7 = 0x1000
    rng = np.random.default_rng(77)
    n = int(np.prod(shape))
    s0 = (2 * rng.integers(0, 2, n) - 1).astype(np.int8)
    key = rng.integers(0, 2**32, 2, dtype=np.uint64).astype(np.uint32)
    raw, s_gpu, running = _run_gpu(cuda, shape, sched, beta, 0.0, s0, key, 12, mode | philox7, k_inline,
                                   chunks=[5, 7])
    s_ref = s0.copy()
    e, m, aux, run = oracle.ising_msc_run(s_ref, shape, key, beta, 0.0, sched, 12, rounds=7)
    np.testing.assert_array_equal(s_gpu, s_ref)
    np.testing.assert_array_equal(raw["Eb"], e)
    np.testing.assert_array_equal(raw["M"], m)
    np.testing.assert_array_equal(raw["aux"], aux)
    s10 = s0.copy()
    e10, _, _, _ = oracle.ising_msc_run(s10, shape, key, beta, 0.0, sched, 12)
    assert not np.array_equal(e, e10)
