"""critmc_ising_msc_run_batch: separately allocated chains with their own keys,
sweep counters and acceptance tables in one call give, bit for bit, what
critmc_ising_msc_run gives for each chain alone (and the oracle's replay)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import oracle
from critmc_b200 import Ising, _lib
from critmc_b200.device import empty_bytes, ptr, stream_handle, to_dev, to_host
from critmc_b200.lattice import hypercubic
from critmc_b200.layout import msc_pack, msc_unpack

pytestmark = pytest.mark.gpu


class MscChain(ctypes.Structure):
    _fields_ = [("spins", ctypes.c_void_p), ("running", ctypes.c_void_p), ("e_out", ctypes.c_void_p),
                ("m_out", ctypes.c_void_p), ("aux_out", ctypes.c_void_p), ("key", ctypes.c_uint32 * 2),
                ("sweep0", ctypes.c_uint32), ("table", ctypes.c_int32)]


@pytest.mark.parametrize("shape,sched,mode", [
    ((256, 64), [[0, 1]], 3),
    ((128, 32), [[0, 2], [2, 1]], 1),
    ((64, 8, 6), [[2, 1]], 0),
])
def test_batch_equals_chains_alone(cuda, shape, sched, mode):
    rng = np.random.default_rng(11)
    model = Ising(hypercubic(shape))
    betas = (0.40, 0.4406868, 0.47) if len(shape) == 2 else (0.21, 0.2216546, 0.23)
    tables = np.ascontiguousarray(np.stack([model.tables(b)[0] for b in betas]))
    n_chains, n_meas = 5, 7
    sched = np.asarray(sched, np.int64)
    per = int(sched[:, 1].sum())
    states = [(2 * rng.integers(0, 2, model.n_sites) - 1).astype(np.int8) for _ in range(n_chains)]
    keys = rng.integers(0, 2**32, (n_chains, 2), dtype=np.uint64).astype(np.uint32)
    sweep0 = [int(x) for x in rng.integers(0, 1000, n_chains)]
    table = [c % 3 for c in range(n_chains)]
    dims = tuple(shape) + (1,) * (3 - len(shape))
    st = stream_handle(cuda)

    def fresh():
        return ([to_dev(msc_pack(s, shape), cuda) for s in states],
                [torch.tensor([[model.bond_energy(s), int(s.astype(np.int64).sum())]], dtype=torch.int64,
                              device=cuda) for s in states])

    # alone: one critmc_ising_msc_run per chain
    a_w, a_run = fresh()
    alone = []
    for c in range(n_chains):
        e = torch.empty((1, 2 * n_meas), dtype=torch.int64, device=cuda)
        m, aux = torch.empty_like(e), torch.empty((1, 2 * n_meas, 4), dtype=torch.int64, device=cuda)
        scratch = empty_bytes(_lib.lib().critmc_ising_msc_scratch_bytes(1, 2 * n_meas), cuda)
        tab = np.ascontiguousarray(tables[table[c]][None])
        _lib.call("critmc_ising_msc_run", ptr(a_w[c]), len(shape), *dims, 1, keys[c].ctypes.data, tab.ctypes.data, 1,
                  sweep0[c], sched.ctypes.data, len(sched), 2 * n_meas, ptr(a_run[c]), ptr(e), ptr(m), ptr(aux),
                  ptr(scratch), mode, 8, st)
        alone.append((e, m, aux))
    # batch: two calls in a row
    b_w, b_run = fresh()
    outs = [[torch.empty(n_meas, dtype=torch.int64, device=cuda) for _ in range(3)] for _ in range(n_chains)]
    auxs = [[torch.empty((n_meas, 4), dtype=torch.int64, device=cuda) for _ in range(2)] for _ in range(n_chains)]
    got = [[] for _ in range(n_chains)]
    scratch = empty_bytes(_lib.lib().critmc_ising_msc_batch_scratch_bytes(n_chains, n_meas), cuda)
    for call in range(2):
        arr = (MscChain * n_chains)()
        for c in range(n_chains):
            e = torch.empty(n_meas, dtype=torch.int64, device=cuda)
            m = torch.empty_like(e)
            aux = torch.empty((n_meas, 4), dtype=torch.int64, device=cuda)
            arr[c].spins, arr[c].running = ptr(b_w[c]), ptr(b_run[c])
            arr[c].e_out, arr[c].m_out, arr[c].aux_out = ptr(e), ptr(m), ptr(aux)
            arr[c].key[0], arr[c].key[1] = int(keys[c][0]), int(keys[c][1])
            arr[c].sweep0 = sweep0[c] + call * n_meas * per
            arr[c].table = table[c]
            got[c].append((e, m, aux))
        _lib.call("critmc_ising_msc_run_batch", ctypes.cast(arr, ctypes.c_void_p), n_chains, len(shape), *dims,
                  tables.ctypes.data, 3, sched.ctypes.data, len(sched), n_meas, ptr(scratch), mode, st)
    torch.cuda.synchronize(cuda)
    for c in range(n_chains):
        e = np.concatenate([to_host(x[0]) for x in got[c]])
        m = np.concatenate([to_host(x[1]) for x in got[c]])
        aux = np.concatenate([to_host(x[2]) for x in got[c]])
        np.testing.assert_array_equal(e, to_host(alone[c][0])[0], err_msg=f"chain {c} E_b")
        np.testing.assert_array_equal(m, to_host(alone[c][1])[0], err_msg=f"chain {c} M")
        np.testing.assert_array_equal(aux, to_host(alone[c][2])[0], err_msg=f"chain {c} aux")
        np.testing.assert_array_equal(to_host(b_w[c]), to_host(a_w[c]), err_msg=f"chain {c} spins")
        np.testing.assert_array_equal(to_host(b_run[c]), to_host(a_run[c]))
    # and one chain against the oracle's replay
    c = 3
    s_ref = states[c].copy()
    er, mr, _, _ = oracle.ising_msc_run(s_ref, shape, keys[c], betas[table[c]], 0.0, sched, 2 * n_meas,
                                        sweep0=sweep0[c])
    np.testing.assert_array_equal(to_host(alone[c][0])[0], er)
    np.testing.assert_array_equal(msc_unpack(to_host(b_w[c], np.uint32), shape), s_ref)


def test_batch_rejects_bad_arguments(cuda):
    lib = _lib.lib()
    arr = (MscChain * 1)()
    sched = np.array([[0, 1]], np.int64)
    tables = np.zeros((1, 2, 2, 16), np.uint32)
    st = lib.critmc_ising_msc_run_batch(ctypes.cast(arr, ctypes.c_void_p), 17, 2, 64, 4, 1, tables.ctypes.data, 1,
                                        sched.ctypes.data, 1, 3, None, 0, None)
    assert st == -1
    st = lib.critmc_ising_msc_run_batch(ctypes.cast(arr, ctypes.c_void_p), 1, 2, 64, 4, 1, tables.ctypes.data, 1,
                                        sched.ctypes.data, 1, 3, ctypes.c_void_p(16), 0, None)
    assert st == -1 and "null" in _lib.last_error()
