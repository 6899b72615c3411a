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
    s = np.ascontiguousarray(state, dtype=np.int8).copy()
    order = initial_order(s, q)
    ln_g = np.zeros(levels)
    hist = np.zeros(levels, dtype=np.int64)
    seen = np.zeros(levels, dtype=bool)
    cps = list(sorted(checkpoints)) if checkpoints is not None else []
    saved, stages = [], []
    check_moves = max(1, int(check_sweeps) * n_sites)
    ln_f, mode_1t, n_lev, t, trials = 1.0, False, 0.0, 0, 0
    while True:
        block = check_moves
        if cps and cps[0] - t < block:
            block = int(cps[0] - t)
        if block > 0:
            idx, trials, _, _ = oracle.fh_run(0, s, shape, q, key, idx, order, ln_g, hist, window, trials, ln_f,
                                              n_lev, mode_1t, 0, block)
            t += block
        seen |= hist > 0
        if mode_1t:
            ln_f = n_lev / t
        while cps and cps[0] <= t:
            saved.append((int(cps.pop(0)), float(ln_f), ln_g.copy()))
        if not mode_1t:
            h = hist[seen]
            ok = h.min() > 0 if criterion == "visit" else h.min() >= flatness * h.mean()
            if ok:
                stages.append({"ln_f": ln_f, "trials": t})
                ln_f /= 2.0
                hist[:] = 0
                if one_over_t and ln_f < seen.sum() / t:
                    mode_1t = True
                    n_lev = float(seen.sum())
                    ln_f = n_lev / t
        if ln_f < ln_f_final or t >= max_trials:
            break
    saved.extend((int(c), float(ln_f), ln_g.copy()) for c in cps)
    return {"ln_g": ln_g, "visited": seen, "trials": t, "ln_f": ln_f, "stages": stages, "checkpoints": saved,
            "state": s, "idx": idx}


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
