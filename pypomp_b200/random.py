"""Random keys for the CUDA particle filters.

The reference takes ``jax.random`` keys and splits them on the host
(``pypomp/core/pomp.py:391-408`` ``_update_fresh_key``;
``estimation_mixin.py:188-190`` one key per (parameter set, replicate)).
JAX is not a dependency here, so a key is a 64-bit integer and ``split``
derives new keys with SplitMix64 (Steele, Lea & Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014).  Each filter's key becomes the
Philox4x32-10 key of its noise stream (``include/ppf_philox.h``).
"""

from __future__ import annotations

import numpy as np

_M64 = (1 << 64) - 1


def _splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & _M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def key(seed: int) -> np.ndarray:
    """A key from an integer seed (``jax.random.key`` analogue)."""
    return np.asarray(_splitmix64(int(seed) & _M64), dtype=np.uint64)


def split(k, num: int = 2) -> np.ndarray:
    """``num`` new keys derived from ``k`` (``jax.random.split`` analogue)."""
    k = int(np.asarray(k, dtype=np.uint64))
    return np.asarray([_splitmix64(k ^ _splitmix64(i + 1)) for i in range(num)], dtype=np.uint64)


def as_key(k) -> np.ndarray:
    """Accept an int seed or a key array; return a uint64 key."""
    if isinstance(k, (int, np.integer)) and not isinstance(k, np.uint64):
        return key(int(k))
    return np.asarray(k, dtype=np.uint64)
