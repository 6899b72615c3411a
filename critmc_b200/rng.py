"""Seeding.

Host-side randomness (initial configurations, couplings) flows through a
numpy ``Generator(PCG64DXSM)`` made exactly as critmc does
(``src/critmc/rng.py:28-71``: ``SeedSequence(entropy=seed, spawn_key=keys)``
with CRC-32 keys for non-integers), so a seed reproduces critmc's initial
state.  The device kernels draw from Philox4x32-10; each chain's 64-bit
Philox key is drawn from that same Generator, so ``(seed, *keys)`` still
names a stream reproducibly and independently of batching.
"""

from __future__ import annotations

import zlib
from collections.abc import Hashable

import numpy as np

__all__ = ["seed_sequence", "make_rng", "spawn_rngs", "philox_key"]


def _key_to_int(key: Hashable) -> int:
    if isinstance(key, (bool, np.bool_)):
        return int(key)
    if isinstance(key, (int, np.integer)):
        if key < 0:
            raise ValueError("integer stream keys must be non-negative")
        return int(key)
    text = key if isinstance(key, str) else repr(key)
    return zlib.crc32(text.encode("utf-8"))


def seed_sequence(seed: int | None, *keys: Hashable) -> np.random.SeedSequence:
    return np.random.SeedSequence(entropy=seed, spawn_key=tuple(_key_to_int(k) for k in keys))


def make_rng(seed=None, *keys: Hashable) -> np.random.Generator:
    if isinstance(seed, np.random.Generator):
        if keys:
            raise ValueError("stream keys cannot be applied to an existing Generator")
        return seed
    if isinstance(seed, np.random.SeedSequence):
        ss = seed
        if keys:
            ss = np.random.SeedSequence(
                entropy=ss.entropy, spawn_key=ss.spawn_key + tuple(_key_to_int(k) for k in keys)
            )
    else:
        ss = seed_sequence(seed, *keys)
    return np.random.Generator(np.random.PCG64DXSM(ss))


def spawn_rngs(seed: int | None, n: int, *keys: Hashable) -> list[np.random.Generator]:
    return [make_rng(seed, *keys, i) for i in range(n)]


def philox_key(rng: np.random.Generator) -> np.ndarray:
    """Two uint32 words of Philox key drawn from ``rng``."""
    return rng.integers(0, 1 << 32, size=2, dtype=np.uint64).astype(np.uint32)
