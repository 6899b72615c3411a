"""CPU oracle of the critmc_b200 kernels.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``.  The library itself never calls
it.  ``liboracle.so`` is a plain-C restatement of critmc's numba kernels
(file:line citations in each ``oracle_*.c``) driven by the same Philox
streams as the GPU kernels, so it reproduces their results bit for bit
(integer models) or to rounding (O(n) models).
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_lib = None


def build() -> Path:
    """Compile ``liboracle.so`` with the Makefile next to this file."""
    res = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        srcs = list(HERE.glob("oracle_*.c")) + [HERE / "oracle.h",
                                                 HERE.parent / "critmc_b200" / "csrc" / "fpmath.h"]
        if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max(p.stat().st_mtime for p in srcs):
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_U32 = ctypes.c_uint32


def _declare(L: ctypes.CDLL) -> None:
    L.oracle_philox.argtypes = [_P, _P, _P]
    L.oracle_philox.restype = None
    L.oracle_ising_table.argtypes = [_I, _I, _D, _D, _P, _P]
    L.oracle_ising_table.restype = _I
    L.oracle_ising_bond_energy.argtypes = [_P, _I, _I, _I, _I]
    L.oracle_ising_bond_energy.restype = ctypes.c_int64
    L.oracle_ising_msc_run.argtypes = [_P, _I, _I, _I, _I, _P, _P, _U32, _P, _I, _I, _P, _P, _P, _P]
    L.oracle_ising_msc_run.restype = _I
    L.oracle_ising_msc_run_rounds.argtypes = [_P, _I, _I, _I, _I, _P, _P, _U32, _P, _I, _I, _P, _P, _P, _P, _I]
    L.oracle_ising_msc_run_rounds.restype = _I
    L.oracle_philox_rounds.argtypes = [_P, _P, _P, _I]
    L.oracle_philox_rounds.restype = None
    L.oracle_ising_byte_run.argtypes = [_P, _I, _I, _I, _I, _P, _P, _U32, _P, _I, _I, _P, _P, _P, _P]
    L.oracle_ising_byte_run.restype = _I
    L.oracle_potts_tables.argtypes = [_I, _D, _P, _P]
    L.oracle_potts_tables.restype = _I
    L.oracle_potts_run.argtypes = [_P, _I, _I, _I, _I, _I, _P, _D, _U32, _P, _I, _I, _P, _P, _P, _P, _P]
    L.oracle_potts_run.restype = _I
    L.oracle_on_run.argtypes = [_P, _I, _I, _I, _I, _I, _P, _D, _D, _U32, _P, _I, _I, _P, _P, _P, _P, _P]
    L.oracle_on_run.restype = _I
    L.oracle_cluster_update.argtypes = [_P, _I, _I, _I, _I, _I, _P, _D, _I, _U32, _P, _P, _P, _P]
    L.oracle_cluster_update.restype = _I
    L.oracle_on_cluster_update.argtypes = [_P, _I, _I, _I, _I, _I, _P, _D, _I, _U32, _P]
    L.oracle_on_cluster_update.restype = _I
    L.oracle_fh_run.argtypes = [_I, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _I, _P, _D, _D, _I,
                                ctypes.c_uint64, ctypes.c_int64, _I, _P, _P]
    L.oracle_fh_run.restype = _I
    L.oracle_fh_descend.argtypes = [_P, _I, _I, _I, _I, _I, _P, _P, _P, _I, _I, ctypes.c_int64]
    L.oracle_fh_descend.restype = ctypes.c_int64
    L.oracle_ea_pt_run.argtypes = [_P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _I, _P, _P, _U32, _I, _I, _I,
                                   _P, _P, _P, _P, _P]
    L.oracle_ea_pt_run.restype = _I
    L.critmc_port_pcg_raw.argtypes = [_P, ctypes.c_int64, _P]
    L.critmc_port_pcg_raw.restype = None
    L.critmc_port_ising_run.argtypes = [_P, _P, ctypes.c_int64, _I, _D, _D, _P, _P, _I, _I, _P, _P, _P, _P]
    L.critmc_port_ising_run.restype = _I


def cluster_update(lay: np.ndarray, shape, q: int, key, beta: float, algo: int, sweep: int,
                   stats: np.ndarray | None = None):
    """One Wolff (algo 3) or SW (4) update of int8 values in the colour-major layout (in place).

    Returns (dE, dM, counts_delta, stats): Ising dE of E_b, Potts dE of E and the
    change of the state counts.
    """
    lay8 = np.ascontiguousarray(lay, dtype=np.int8)
    flat = lay8.reshape(-1)
    lx, ly, lz = _dims(shape)
    k = np.ascontiguousarray(key, dtype=np.uint32).reshape(2)
    de = ctypes.c_int64(0)
    dm = ctypes.c_int64(0)
    cd = np.zeros(max(q, 1), dtype=np.int64)
    st = np.zeros(3, dtype=np.int64) if stats is None else stats
    rc = lib().oracle_cluster_update(_ptr(flat), len(shape), lx, ly, lz, q, _ptr(k), float(beta), algo, sweep,
                                     ctypes.byref(de), ctypes.byref(dm), _ptr(cd), _ptr(st))
    if rc:
        raise MemoryError("oracle_cluster_update")
    lay[...] = flat.reshape(lay.shape)
    return de.value, dm.value, cd[:q] if q else None, st


def on_cluster_update(comps: np.ndarray, shape, key, beta: float, algo: int, sweep: int,
                      stats: np.ndarray | None = None) -> np.ndarray:
    """One O(n) Wolff (3) / SW (4) update of float32 components [n][N] (colour-major, in place).

    Returns the stats triple (Wolff size added; SW sum |C|^2, cluster count).
    """
    lx, ly, lz = _dims(shape)
    if comps.dtype != np.float32 or not comps.flags["C_CONTIGUOUS"]:
        raise TypeError("comps is updated in place: pass a C-contiguous float32 array")
    k = np.ascontiguousarray(key, dtype=np.uint32).reshape(2)
    st = np.zeros(3, dtype=np.int64) if stats is None else stats
    rc = lib().oracle_on_cluster_update(_ptr(comps), len(shape), lx, ly, lz, comps.shape[0], _ptr(k), float(beta),
                                        algo, sweep, _ptr(st))
    if rc != 0:
        raise MemoryError("oracle_on_cluster_update")
    return st


def fh_descend(s: np.ndarray, shape, q: int, key, idx: int, order: np.ndarray, window, max_steps: int):
    """Greedy descent of one walker into its window (arrays in place); returns (idx, steps or -1)."""
    lx, ly, lz = _dims(shape)
    if s.dtype != np.int8 or order.dtype != np.int64 or not (s.flags["C_CONTIGUOUS"] and order.flags["C_CONTIGUOUS"]):
        raise TypeError("s (int8) and order (int64) are updated in place")
    k = np.ascontiguousarray(key, dtype=np.uint32).reshape(2)
    i = ctypes.c_int64(idx)
    steps = lib().oracle_fh_descend(_ptr(s), len(shape), lx, ly, lz, q, _ptr(k), ctypes.byref(i), _ptr(order),
                                    int(window[0]), int(window[1]), int(max_steps))
    return i.value, int(steps)


def fh_run(mode: int, s: np.ndarray, shape, q: int, key, idx: int, order: np.ndarray, lng: np.ndarray,
           hist: np.ndarray, window, trials: int, ln_f: float, n_levels: float, one_over_t: bool, t_base: int,
           moves: int, n_meas: int = 1):
    """One walker's Wang-Landau (mode 0) or multicanonical (1) moves; arrays updated in place.

    Returns (idx, trials, idx_out, order_out).
    """
    lx, ly, lz = _dims(shape)
    k = np.ascontiguousarray(key, dtype=np.uint32).reshape(2)
    i = ctypes.c_int64(idx)
    t = ctypes.c_uint64(trials)
    io = np.zeros(max(n_meas, 1), dtype=np.int64)
    oo = np.zeros(max(n_meas, 1), dtype=np.int64)
    for a, dt in ((s, np.int8), (order, np.int64), (lng, np.float64), (hist, np.int64)):
        if a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
            raise TypeError("arrays are updated in place: pass contiguous arrays of the right dtype")
    lib().oracle_fh_run(mode, _ptr(s), len(shape), lx, ly, lz, q, _ptr(k), ctypes.byref(i), _ptr(order),
                        _ptr(lng), _ptr(hist), int(window[0]), int(window[1]), ctypes.byref(t), float(ln_f),
                        float(n_levels), int(one_over_t), ctypes.c_uint64(t_base), int(moves), int(n_meas),
                        _ptr(io), _ptr(oo))
    return i.value, t.value, io[:n_meas], oo[:n_meas]


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def philox_rounds(ctr, key, rounds: int) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox_rounds(_ptr(c), _ptr(k), _ptr(out), int(rounds))
    return out


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox(_ptr(c), _ptr(k), _ptr(out))
    return out


def ising_table(algo: int, z: int, beta: float, h: float) -> np.ndarray:
    """``(2, 16)`` uint32: kind row then thr row."""
    kind = np.zeros(16, dtype=np.uint32)
    thr = np.zeros(16, dtype=np.uint32)
    if lib().oracle_ising_table(algo, z, beta, h, _ptr(kind), _ptr(thr)) != 0:
        raise ValueError("unsupported algorithm")
    return np.stack([kind, thr])


def ising_bond_energy(s: np.ndarray, shape: tuple[int, ...]) -> int:
    dims = tuple(shape) + (1,) * (3 - len(shape))
    s8 = np.ascontiguousarray(s, dtype=np.int8)
    return int(lib().oracle_ising_bond_energy(_ptr(s8), len(shape), *dims))


def ising_msc_run(s, shape, key, beta, h, schedule, n_meas, sweep0=0, running=None, rounds=10):
    """Replay the MSC checkerboard sweeps on ``s`` (int8, reference site order, modified).

    ``rounds``: Philox rounds of the acceptance planes (10, or the optional 7).
    Returns ``(e_b, m, aux, running)``.
    """
    s8 = s if (isinstance(s, np.ndarray) and s.dtype == np.int8 and s.flags["C_CONTIGUOUS"]) else None
    if s8 is None:
        raise TypeError("s must be a C-contiguous int8 array (it is updated in place)")
    dims = tuple(shape) + (1,) * (3 - len(shape))
    z = 2 * len(shape)
    tables = np.concatenate([ising_table(0, z, beta, h).ravel(), ising_table(2, z, beta, h).ravel()])
    tables = np.ascontiguousarray(tables, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    if running is None:
        running = np.array([ising_bond_energy(s8, shape), int(s8.astype(np.int64).sum())], dtype=np.int64)
    running = np.ascontiguousarray(running, dtype=np.int64).copy()
    e = np.zeros(n_meas, dtype=np.int64)
    m = np.zeros(n_meas, dtype=np.int64)
    aux = np.zeros((n_meas, 4), dtype=np.int64)
    rc = lib().oracle_ising_msc_run_rounds(
        _ptr(s8), len(shape), *dims, _ptr(k), _ptr(tables), sweep0, _ptr(sched), len(sched), n_meas,
        _ptr(running), _ptr(e), _ptr(m), _ptr(aux), int(rounds),
    )
    if rc != 0:
        raise ValueError(f"oracle_ising_msc_run failed ({rc})")
    return e, m, aux, running


def _dims(shape):
    return tuple(shape) + (1,) * (3 - len(shape))


def ising_byte_run(s, shape, key, beta, h, schedule, n_meas, sweep0=0, running=None):
    """Replay the int8 checkerboard sweeps on ``s`` (int8, critmc order, modified in place)."""
    if not (isinstance(s, np.ndarray) and s.dtype == np.int8 and s.flags["C_CONTIGUOUS"]):
        raise TypeError("s must be a C-contiguous int8 array (it is updated in place)")
    z = 2 * len(shape)
    tables = np.ascontiguousarray(
        np.concatenate([ising_table(0, z, beta, h).ravel(), ising_table(2, z, beta, h).ravel()]),
        dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    if running is None:
        running = np.array([ising_bond_energy(s, shape), int(s.astype(np.int64).sum())], dtype=np.int64)
    running = np.ascontiguousarray(running, dtype=np.int64).copy()
    e = np.zeros(n_meas, dtype=np.int64)
    m = np.zeros(n_meas, dtype=np.int64)
    aux = np.zeros((n_meas, 4), dtype=np.int64)
    rc = lib().oracle_ising_byte_run(_ptr(s), len(shape), *_dims(shape), _ptr(k), _ptr(tables), sweep0,
                                     _ptr(sched), len(sched), n_meas, _ptr(running), _ptr(e), _ptr(m),
                                     _ptr(aux))
    if rc != 0:
        raise ValueError(f"oracle_ising_byte_run failed ({rc})")
    return e, m, aux, running


def potts_tables(z: int, beta: float):
    b = np.zeros(8, dtype=np.uint64)
    w = np.zeros(8, dtype=np.uint64)
    lib().oracle_potts_tables(z, beta, _ptr(b), _ptr(w))
    return b, w


def potts_energy(s, shape) -> int:
    """E = -#satisfied bonds (critmc kernels/potts.py:28-34)."""
    a = np.asarray(s).reshape(tuple(reversed(tuple(shape))))
    e = 0
    for ax in range(a.ndim):
        e -= int(np.sum(a == np.roll(a, -1, axis=ax)))
    return e


def potts_run(s, shape, q, key, beta, schedule, n_meas, sweep0=0, energy=None, counts=None):
    """Replay the Potts checkerboard sweeps on ``s`` (int8 states, modified in place)."""
    if not (isinstance(s, np.ndarray) and s.dtype == np.int8 and s.flags["C_CONTIGUOUS"]):
        raise TypeError("s must be a C-contiguous int8 array (it is updated in place)")
    k = np.ascontiguousarray(key, dtype=np.uint32)
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    en = np.array([potts_energy(s, shape) if energy is None else energy], dtype=np.int64)
    cnt = (np.bincount(s.astype(np.int64), minlength=q) if counts is None else np.array(counts)).astype(np.int64)
    cnt = np.ascontiguousarray(cnt)
    e = np.zeros(n_meas, dtype=np.int64)
    co = np.zeros((n_meas, q), dtype=np.int64)
    aux = np.zeros((n_meas, 4), dtype=np.int64)
    rc = lib().oracle_potts_run(_ptr(s), len(shape), *_dims(shape), q, _ptr(k), beta, sweep0, _ptr(sched),
                                len(sched), n_meas, _ptr(en), _ptr(cnt), _ptr(e), _ptr(co), _ptr(aux))
    if rc != 0:
        raise ValueError(f"oracle_potts_run failed ({rc})")
    return e, co, aux, int(en[0]), cnt


def on_run(s, shape, n, key, beta, step, schedule, n_meas, sweep0=0):
    """Replay the O(n) checkerboard sweeps on ``s`` (float32 (N, n), critmc order, in place).

    Returns ``(E, M, stiff_c, stiff_s, aux)`` like critmc's ``ON.advance``.
    """
    if not (isinstance(s, np.ndarray) and s.dtype == np.float32 and s.flags["C_CONTIGUOUS"]):
        raise TypeError("s must be a C-contiguous float32 array (it is updated in place)")
    dim = len(shape)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    e = np.zeros(n_meas)
    m = np.zeros((n_meas, n))
    sc = np.zeros((n_meas, dim))
    ss = np.zeros((n_meas, dim))
    aux = np.zeros((n_meas, 4), dtype=np.int64)
    rc = lib().oracle_on_run(_ptr(s), dim, *_dims(shape), n, _ptr(k), beta, step, sweep0, _ptr(sched),
                             len(sched), n_meas, _ptr(e), _ptr(m), _ptr(sc), _ptr(ss), _ptr(aux))
    if rc != 0:
        raise ValueError(f"oracle_on_run failed ({rc})")
    return e, m, sc, ss, aux


def ea_pt_run(spins, couplings, shape, keys, betas, swap_thr, perm, labels, n_steps, n_bins,
              t0=0, sweeps_per_step=1):
    """Replay parallel tempering of one +-J sample (critmc pt_run layout, arrays updated in place).

    spins: int8 (2, m, N); couplings: float64 (dim N,); keys: uint32 (2, 2);
    perm, labels: int32 (2, m).  Returns (acc, swap_acc, swap_try, label_hist, trips).
    """
    m = spins.shape[1]
    for a, dt in ((spins, np.int8), (perm, np.int32), (labels, np.int32)):
        if not (isinstance(a, np.ndarray) and a.dtype == dt and a.flags["C_CONTIGUOUS"]):
            raise TypeError("spins/perm/labels must be C-contiguous int8/int32 arrays")
    J = np.ascontiguousarray(couplings, dtype=np.float64)
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    b = np.ascontiguousarray(betas, dtype=np.float64)
    st = np.ascontiguousarray(swap_thr, dtype=np.uint32)
    acc = np.zeros((n_bins, m, 7))
    sa = np.zeros(m - 1, dtype=np.int64)
    stry = np.zeros(m - 1, dtype=np.int64)
    lh = np.zeros((m, 2), dtype=np.int64)
    tr = np.zeros(2, dtype=np.int64)
    rc = lib().oracle_ea_pt_run(_ptr(spins), _ptr(J), len(shape), *_dims(shape), m, _ptr(k), _ptr(b),
                                _ptr(st), st.shape[1], _ptr(perm), _ptr(labels), t0, n_steps, n_bins,
                                sweeps_per_step, _ptr(acc), _ptr(sa), _ptr(stry), _ptr(lh), _ptr(tr))
    if rc != 0:
        raise ValueError(f"oracle_ea_pt_run failed ({rc})")
    return acc, sa, stry, lh, tr


def pcg_words(state: dict) -> np.ndarray:
    """numpy PCG64DXSM state dict -> (state hi, state lo, inc hi, inc lo)."""
    st = state["state"] if "inc" not in state else state
    s, inc = int(st["state"]), int(st["inc"])
    m = (1 << 64) - 1
    return np.array([s >> 64, s & m, inc >> 64, inc & m], dtype=np.uint64)


def pcg_raw(words: np.ndarray, n: int) -> np.ndarray:
    """The next n raw outputs of the C PCG64DXSM (words updated in place)."""
    out = np.zeros(n, dtype=np.uint64)
    lib().critmc_port_pcg_raw(_ptr(words), n, _ptr(out))
    return out


def critmc_ising_run(s, nbr, words, beta, h, schedule, n_meas, running=None):
    """critmc's CPU Ising ``run`` (typewriter Metropolis / heat bath) restated in C.

    ``s`` int8 spins in critmc's site order (updated), ``nbr`` critmc's int64
    (N, z) neighbour table, ``words`` the Generator state (``pcg_words``,
    updated).  Returns ``(e_b, m, aux, running)`` like the GPU entry points.
    """
    if not (isinstance(s, np.ndarray) and s.dtype == np.int8 and s.flags["C_CONTIGUOUS"]):
        raise TypeError("s must be a C-contiguous int8 array (it is updated in place)")
    nb = np.ascontiguousarray(nbr, dtype=np.int64)
    n, z = nb.shape
    sched = np.ascontiguousarray(schedule, dtype=np.int64).reshape(-1, 2)
    if running is None:
        i = np.arange(n)
        running = np.array([-int(sum(int(np.dot(s[i].astype(np.int64), s[nb[:, 2 * a]].astype(np.int64)))
                                     for a in range(z // 2))), int(s.astype(np.int64).sum())], dtype=np.int64)
    running = np.ascontiguousarray(running, dtype=np.int64).copy()
    e = np.zeros(n_meas, dtype=np.int64)
    m = np.zeros(n_meas, dtype=np.int64)
    aux = np.zeros((n_meas, 4), dtype=np.int64)
    rc = lib().critmc_port_ising_run(_ptr(s), _ptr(nb), n, z, float(beta), float(h), _ptr(words), _ptr(sched),
                                     len(sched), n_meas, _ptr(running), _ptr(e), _ptr(m), _ptr(aux))
    if rc != 0:
        raise ValueError(f"critmc_port_ising_run failed ({rc})")
    return e, m, aux, running
