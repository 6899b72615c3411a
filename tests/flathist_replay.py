"""CPU replay of the flat-histogram schedules through the oracle (test infrastructure).

``replay_wang_landau`` restates the host schedule of critmc's
``WangLandau.run`` (src/critmc/flathist.py:247-320) around ``oracle.fh_run``,
so a GPU run started from the same configuration, level and key must give
the same ``ln g``, histogram, stages and trial count bit for bit.
"""

from __future__ import annotations

import numpy as np

import oracle


def initial_order(state: np.ndarray, q: int) -> np.ndarray:
    if q == 0:
        return np.array([int(state.astype(np.int64).sum())], dtype=np.int64)
    return np.bincount(state.astype(np.int64), minlength=q).astype(np.int64)


def replay_wang_landau(shape, q: int, state: np.ndarray, key, idx: int, window, levels: int, n_sites: int,
                       ln_f_final: float, *, one_over_t: bool = True, check_sweeps: int = 100,
                       flatness: float = 0.8, criterion: str = "flat", max_trials: float = 1e12,
                       checkpoints=None) -> dict:
    """One walker through critmc's Wang-Landau schedule, the moves on the oracle.

    Blocks of ``check_sweeps`` N moves (cut short at checkpoints); after each:
    the levels visited so far, ln f = n_levels / t once in 1/t mode, copies of
    ln g at passed checkpoints, and (before 1/t mode) the flatness or visit
    test, whose success records a stage, halves ln f, clears the histogram and
    may switch to 1/t mode when ln f < n_seen / t.  Stops at ln f < ln_f_final
    or ``max_trials``; later checkpoints get the final ln g.
    """
    spins = np.ascontiguousarray(state, dtype=np.int8).copy()
    order = initial_order(spins, q)
    ln_g = np.zeros(levels)
    visits = np.zeros(levels, dtype=np.int64)
    seen = np.zeros(levels, dtype=bool)
    marks = sorted(checkpoints) if checkpoints is not None else []
    kept, stages = [], []
    ln_f, inverse_t, n_levels, t, trials = 1.0, False, 0.0, 0, 0
    while ln_f >= ln_f_final and t < max_trials:
        step = max(1, int(check_sweeps) * n_sites)
        if marks:
            step = min(step, int(marks[0] - t))
        if step > 0:
            idx, trials, _, _ = oracle.fh_run(0, spins, shape, q, key, idx, order, ln_g, visits, window, trials,
                                              ln_f, n_levels, inverse_t, 0, step)
            t += step
        seen = seen | (visits > 0)
        if inverse_t:
            ln_f = n_levels / t
        while marks and marks[0] <= t:
            kept.append((int(marks.pop(0)), float(ln_f), ln_g.copy()))
        if inverse_t:
            continue
        counts = visits[seen]
        passed = counts.min() > 0 if criterion == "visit" else counts.min() >= flatness * counts.mean()
        if not passed:
            continue
        stages.append({"ln_f": ln_f, "trials": t})
        ln_f = ln_f / 2.0
        visits[:] = 0
        if one_over_t and ln_f < seen.sum() / t:
            inverse_t, n_levels = True, float(seen.sum())
            ln_f = n_levels / t
    kept += [(int(m), float(ln_f), ln_g.copy()) for m in marks]
    return {"ln_g": ln_g, "visited": seen, "trials": t, "ln_f": ln_f, "stages": stages, "checkpoints": kept,
            "state": spins, "idx": idx}


def replay_multicanonical(shape, q: int, state: np.ndarray, key, idx: int, window, ln_w: np.ndarray,
                          moves: int, n_meas: int, n_therm: int = 0) -> dict:
    s = np.ascontiguousarray(state, dtype=np.int8).copy()
    order = initial_order(s, q)
    lw = np.ascontiguousarray(ln_w, dtype=np.float64).copy()
    trials = 0
    if n_therm:
        scratch = np.zeros(lw.size, dtype=np.int64)
        idx, trials, _, _ = oracle.fh_run(1, s, shape, q, key, idx, order, lw, scratch, window, trials, 0.0, 0.0,
                                          False, 0, moves, n_therm)
    hist = np.zeros(lw.size, dtype=np.int64)
    idx, trials, io, oo = oracle.fh_run(1, s, shape, q, key, idx, order, lw, hist, window, trials, 0.0, 0.0, False,
                                        0, moves, n_meas)
    return {"level_series": io, "order_series": oo, "hist": hist, "state": s, "idx": idx, "trials": trials}


def walk_into_window(model, state: np.ndarray, levels, lo: int, hi: int, rng, max_steps: int = 10**7) -> int:
    """Host restatement of critmc's greedy walk into a level window (flathist.py:96-130).

    A random site gets a proposal (Ising: the flip; Potts: another state drawn
    uniformly) that is kept when the level does not move away from [lo, hi].
    ``state`` is changed in place; returns the level reached.
    """
    nbr = model.lattice.nbr
    level = levels.index(model.energy(state))
    ising = levels.kind == "ising"
    for _ in range(max_steps):
        if lo <= level <= hi:
            return level
        site = int(rng.integers(model.n_sites))
        here = int(state[site])
        around = state[nbr[site]]
        if ising:
            proposal = -here
            new_level = level + here * int(around.astype(np.int64).sum()) // 2
        else:
            proposal = int(rng.integers(levels.q - 1))
            if proposal >= here:
                proposal += 1
            new_level = level + int((around == here).sum()) - int((around == proposal).sum())
        toward = new_level >= level if level < lo else new_level <= level
        if toward:
            state[site] = proposal
            level = new_level
    raise RuntimeError("the walk did not reach the window")
