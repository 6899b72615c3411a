"""Seeding.

Host-side randomness (initial configurations, couplings) comes from a numpy
``Generator(PCG64DXSM)`` seeded the way critmc seeds it
(``src/critmc/rng.py:28-71``): a ``SeedSequence`` whose entropy is the seed and
whose spawn key lists the stream keys, each key turned into an integer (ints
and bools as they are, anything else by the CRC-32 of its text).  A seed with
keys therefore names the same stream, and the same initial state, as in
critmc.  The device kernels draw from Philox4x32-10; each chain's 64-bit Philox
key is drawn from that Generator, so ``(seed, *keys)`` also names the device
stream, independently of batching.
"""

from __future__ import annotations

import zlib
from collections.abc import Hashable

import numpy as np

__all__ = ["seed_sequence", "make_rng", "spawn_rngs", "philox_key"]


def _key_word(key: Hashable) -> int:
    """The spawn-key integer of one stream key."""
    if isinstance(key, (bool, np.bool_, int, np.integer)):
        value = int(key)
        if value < 0:
            raise ValueError(f"integer stream keys must be >= 0, got {value}")
        return value
    label = key if isinstance(key, str) else repr(key)
    return zlib.crc32(label.encode("utf-8"))


def seed_sequence(seed: int | None, *keys: Hashable) -> np.random.SeedSequence:
    """SeedSequence(entropy=seed, spawn_key=the keys' integers)."""
    return np.random.SeedSequence(entropy=seed, spawn_key=tuple(map(_key_word, keys)))


def make_rng(seed=None, *keys: Hashable) -> np.random.Generator:
    """The PCG64DXSM Generator of ``(seed, *keys)``; ``seed`` may be an int, None, a
    SeedSequence (keys extend its spawn key) or a Generator (returned as it is)."""
    if isinstance(seed, np.random.Generator):
        if keys:
            raise ValueError("stream keys need a seed or SeedSequence, not an existing Generator")
        return seed
    if isinstance(seed, np.random.SeedSequence):
        sequence = np.random.SeedSequence(entropy=seed.entropy,
                                          spawn_key=tuple(seed.spawn_key) + tuple(map(_key_word, keys)))
        if not keys:
            sequence = seed
    else:
        sequence = seed_sequence(seed, *keys)
    return np.random.Generator(np.random.PCG64DXSM(sequence))


def spawn_rngs(seed: int | None, n: int, *keys: Hashable) -> list[np.random.Generator]:
    """``n`` independent generators, the i-th keyed by ``(*keys, i)``."""
    return [make_rng(seed, *keys, i) for i in range(n)]


def philox_key(rng: np.random.Generator) -> np.ndarray:
    """Two uint32 words of Philox key drawn from ``rng``."""
    return rng.integers(0, 1 << 32, size=2, dtype=np.uint64).astype(np.uint32)
