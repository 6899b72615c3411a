"""Streaming Gamma-method statistics of many chains' measurement series.

``StreamStats`` keeps, per chain, the sums that determine the autocorrelation
function up to a maximum lag W (count, shift, sum, sum of squares, lag sums,
first and last W values), updated on the device by ``critmc_stream_update``
slice after slice; ``result`` evaluates U. Wolff's Gamma-method (automatic
window, S = 1.5, bias-corrected) from them, as critmc's ``gamma_method``
(src/critmc/stats/autocorr.py:381) does from a full series, provided the
window stays below W (``truncated`` says when it did not).  ``HostStreamStats``
is the same on host arrays (used by the server's summary mode).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import ptr, require_cuda, stream_handle, to_host


def _layout(W: int) -> tuple[int, int, int, int]:
    lag = 4
    head = lag + W
    tail = head + W
    return lag, head, tail, tail + W


def gamma_from_state(st: np.ndarray, W: int, S: float = 1.5) -> dict[str, float]:
    """(mean, error, tau_int, window, truncated) of one chain's streaming state."""
    lag0, head0, tail0, _ = _layout(W)
    n = int(st[0])
    if n == 0:
        return {"n": 0, "mean": float("nan"), "error": float("nan"), "tau_int": float("nan"), "window": 0,
                "truncated": False}
    shift, sy, sy2 = st[1], st[2], st[3]
    lag, head, tail = st[lag0:lag0 + W], st[head0:head0 + W], st[tail0:tail0 + W]
    m = sy / n
    t_max = min(W, n // 2, n - 1)
    gam = np.empty(t_max + 1)
    gam[0] = sy2 / n - m * m
    for t in range(1, t_max + 1):
        a = sy - tail[W - t:].sum()
        b = sy - head[:t].sum()
        gam[t] = (lag[t - 1] - m * (a + b) + (n - t) * m * m) / (n - t)
    mean = float(shift + m)
    if not gam[0] > 0:
        return {"n": n, "mean": mean, "error": 0.0, "tau_int": 0.5, "window": 0, "truncated": False}
    w = np.arange(1, gam.size)
    g_int = np.cumsum(gam[1:]) / gam[0]
    tau_w = np.full(w.size, 1e-300)
    pos = g_int > 0
    with np.errstate(divide="ignore", over="ignore"):
        tau_w[pos] = S / np.log1p(1.0 / g_int[pos])
    tau_w = np.maximum(tau_w, 1e-300)
    g = np.exp(-w / tau_w) - tau_w / np.sqrt(w * float(n))
    hits = np.flatnonzero(g < 0)
    truncated = hits.size == 0 and t_max == W and W < n // 2
    w_opt = int(w[hits[0]]) if hits.size else int(w[-1]) if w.size else 0
    c_f = gam[0] + 2.0 * gam[1:w_opt + 1].sum()
    gam = gam + c_f / n  # bias of the subtracted mean
    c_f = gam[0] + 2.0 * gam[1:w_opt + 1].sum()
    tau = c_f / (2.0 * gam[0])
    err = float(np.sqrt(c_f / n)) if c_f > 0 else float("nan")
    return {"n": n, "mean": mean, "error": err, "tau_int": float(tau), "window": w_opt, "truncated": bool(truncated)}


class StreamStats:
    """Device streaming state for ``n_chains`` series (one observable each)."""

    def __init__(self, n_chains: int, max_lag: int = 256, device=None):
        self.device = require_cuda(device)
        self.n_chains, self.W = int(n_chains), int(max_lag)
        nbytes = _lib.lib().critmc_stream_state_bytes(self.n_chains, self.W)
        if nbytes < 0:
            raise ValueError("need n_chains >= 1 and 1 <= max_lag <= 1024")
        self.state = torch.zeros(nbytes // 8, dtype=torch.float64, device=self.device)

    def update(self, values: torch.Tensor, stream=None) -> None:
        """Append ``values`` ([n_chains, n] int64 or float64, on the device) to every chain's series."""
        if values.dim() == 1:
            values = values.reshape(self.n_chains, -1)
        if values.shape[0] != self.n_chains or values.device != self.device:
            raise ValueError("values must be a device tensor [n_chains, n]")
        if values.dtype not in (torch.int64, torch.float64):
            values = values.to(torch.float64)
        v = values.contiguous()
        _lib.call_on(self.device, "critmc_stream_update", ptr(v), int(v.dtype == torch.float64), self.n_chains,
                     v.shape[1], v.shape[1], ptr(self.state), self.W,
                     stream if stream is not None else stream_handle(self.device))

    def result(self, S: float = 1.5) -> list[dict[str, float]]:
        st = to_host(self.state).reshape(self.n_chains, -1)
        return [gamma_from_state(st[c], self.W, S) for c in range(self.n_chains)]


class HostStreamStats:
    """The same streaming state for one series on the host (numpy)."""

    def __init__(self, max_lag: int = 256):
        self.W = int(max_lag)
        self.state = np.zeros(_layout(self.W)[3])

    def update(self, x) -> None:
        x = np.asarray(x, dtype=np.float64).ravel()
        if x.size == 0:
            return
        W = self.W
        lag0, head0, tail0, _ = _layout(W)
        st = self.state
        n0 = int(st[0])
        if n0 == 0:
            st[1] = x[0]
        y = x - st[1]
        # [last W values (zeros before the start) | new values]: the zeros add nothing
        full = np.concatenate([st[tail0:tail0 + W], y])
        win = np.lib.stride_tricks.sliding_window_view(full, W + 1)  # row j ends with y[j]
        acc = np.zeros(W)
        for j in range(0, y.size, 4096):
            rows = win[j:j + 4096]
            acc += (rows[:, :W] * rows[:, W:]).sum(axis=0)  # column c: lag W - c
        st[lag0:lag0 + W] += acc[::-1]
        st[2] += y.sum()
        st[3] += float(np.dot(y, y))
        if n0 < W:
            k = min(W - n0, y.size)
            st[head0 + n0:head0 + n0 + k] = y[:k]
        st[tail0:tail0 + W] = full[-W:]
        st[0] = n0 + x.size

    def result(self, S: float = 1.5) -> dict[str, float]:
        return gamma_from_state(self.state, self.W, S)
