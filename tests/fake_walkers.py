"""A CPU stand-in for the device walkers of ``critmc_b200.flathist`` (test infrastructure).

It holds the walkers' arrays as CPU tensors and advances them with the oracle,
so the host schedules of ``WangLandau.run`` and ``Multicanonical.run`` can be
checked on a machine without a GPU.  The product never uses it.
"""

from __future__ import annotations

import numpy as np
import torch
from flathist_replay import initial_order

import oracle
from critmc_b200.flathist import EnergyLevels
from critmc_b200.rng import philox_key


class OracleWalkers:
    def __init__(self, model, windows, rngs, device=None):
        self.model = model
        self.levels = EnergyLevels.of(model)
        self.q = 0 if self.levels.kind == "ising" else self.levels.q
        self.n = len(windows)
        self.device = torch.device("cpu")
        self.shape = tuple(model.lattice.shape)
        states, keys, idx, orders = [], [], [], []
        for w, (lo, hi) in enumerate(windows):
            s = np.asarray(model.initial_state("random", rngs[w]), dtype=np.int8)
            k = philox_key(rngs[w])
            o = initial_order(s, self.q)
            i, steps = oracle.fh_descend(s, self.shape, self.q, k, self.levels.index(model.energy(s)), o, (lo, hi),
                                         10**6)
            assert steps >= 0
            states.append(s)
            keys.append(k)
            idx.append(i)
            orders.append(o)
        self.spins = torch.from_numpy(np.stack(states))
        self.keys = torch.from_numpy(np.stack(keys).view(np.int32))
        self.idx = torch.tensor(idx, dtype=torch.int64)
        self.order = torch.from_numpy(np.stack(orders) if self.q else np.concatenate(orders))
        self.window = torch.tensor(np.array(windows, dtype=np.int32))
        self.trials = torch.zeros(self.n, dtype=torch.int64)
        self.hist = torch.zeros((self.n, self.levels.size), dtype=torch.int64)

    def run(self, mode, lng, moves, *, ln_f=None, n_levels=None, one_over_t=None, t_base=None, n_meas=1,
            idx_out=None, order_out=None, memory="auto"):
        for w in range(self.n):
            lo, hi = (int(x) for x in self.window[w])
            if lo < 0:
                continue  # frozen walker, as the kernel skips it
            s = self.spins[w].numpy()
            order = self.order[w].numpy() if self.q else self.order[w:w + 1].numpy()
            i, t, io, oo = oracle.fh_run(
                mode, s, self.shape, self.q, self.keys[w].numpy().view(np.uint32), int(self.idx[w]), order,
                lng[w].numpy(), self.hist[w].numpy(), (lo, hi), int(self.trials[w]),
                float(ln_f[w]) if ln_f is not None else 0.0, float(n_levels[w]) if n_levels is not None else 0.0,
                bool(one_over_t[w]) if one_over_t is not None else False,
                int(t_base[w]) if t_base is not None else 0, moves, n_meas)
            self.idx[w] = i
            self.trials[w] = t
            if idx_out is not None:
                idx_out[w] = torch.from_numpy(io)
                order_out[w] = torch.from_numpy(oo)
