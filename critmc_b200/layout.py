"""Conversions between critmc's site order and the device layouts.

Host arrays use critmc's numbering (first coordinate fastest).  On the
device, binary spins of a checkerboard lattice are stored colour-major and
multi-spin coded (see ``include/critmc_b200.h``):

    words[colour][row][k], row = y + ly*z, bit j of word k holds the colour's
    site x = 2*(32k + j) + p,  p = (colour + y + z) & 1,  bit 1 = spin +1.

Byte and float lattices (Potts, O(n)) use the same colour-major order with
one element per site: ``elem[colour][row][i]`` with ``x = 2i + p``.
"""

from __future__ import annotations

import numpy as np


def _dims3(shape) -> tuple[int, int, int]:
    s = tuple(int(v) for v in shape)
    return (s + (1, 1, 1))[:3]


def checkerboard_order(shape) -> np.ndarray:
    """Site index (critmc order) of every slot of the colour-major layout.

    Returns an int64 array of shape ``(2, rows, lx // 2)``.
    """
    lx, ly, lz = _dims3(shape)
    rows = ly * lz
    r = np.arange(rows)
    y, z = r % ly, r // ly
    i = np.arange(lx // 2)
    out = np.empty((2, rows, lx // 2), dtype=np.int64)
    for c in range(2):
        p = (c + y + z) & 1
        x = 2 * i[None, :] + p[:, None]
        out[c] = x + lx * (y[:, None] + ly * z[:, None])
    return out


def msc_pack(s: np.ndarray, shape) -> np.ndarray:
    """int8 +-1 spins (critmc order) -> uint32 words ``(2, rows, lx // 64)``."""
    lx, ly, lz = _dims3(shape)
    order = checkerboard_order(shape)  # (2, rows, lx/2)
    bits = (np.asarray(s)[order] > 0).astype(np.uint64)  # (2, rows, lx/2)
    bits = bits.reshape(2, ly * lz, lx // 64, 32)
    weights = (np.uint64(1) << np.arange(32, dtype=np.uint64))
    return (bits * weights).sum(axis=-1).astype(np.uint32)


def msc_unpack(words: np.ndarray, shape) -> np.ndarray:
    """uint32 words ``(2, rows, lx // 64)`` -> int8 +-1 spins in critmc order."""
    lx, ly, lz = _dims3(shape)
    w = np.asarray(words, dtype=np.uint32).reshape(2, ly * lz, lx // 64, 1)
    bits = ((w >> np.arange(32, dtype=np.uint32)) & 1).reshape(2, ly * lz, lx // 2)
    order = checkerboard_order(shape)
    s = np.empty(lx * ly * lz, dtype=np.int8)
    s[order.ravel()] = (2 * bits.astype(np.int8) - 1).ravel()
    return s


def cb_pack(values: np.ndarray, shape) -> np.ndarray:
    """Per-site values (critmc order, leading axis = site) -> colour-major array."""
    order = checkerboard_order(shape)
    v = np.asarray(values)
    return np.ascontiguousarray(v[order])


def cb_unpack(packed: np.ndarray, shape) -> np.ndarray:
    """Inverse of :func:`cb_pack`."""
    order = checkerboard_order(shape)
    p = np.asarray(packed)
    out = np.empty((order.size,) + p.shape[3:], dtype=p.dtype)
    out[order.ravel()] = p.reshape((order.size,) + p.shape[3:])
    return out
