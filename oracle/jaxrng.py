"""NumPy restatement of the random-number streams the reference draws from JAX.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped package imports this module;
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may use anything under ``oracle/``.

The reference (pypomp 0.4.10.2) draws every random number through
``jax.random`` (dependency ``jax>=0.5.3``, ``pyproject.toml:28``; JAX is not
installed here and its version is unpinned by the reference).  Its regression
fixtures (``tests/test_regression/*/*.csv``) therefore lock JAX's streams.  To
pin the oracle against those fixtures without JAX, this module restates the
published algorithms JAX uses:

* Threefry-2x32 with 20 rounds (Salmon, Moraes, Dror & Shaw, "Parallel random
  numbers: as easy as 1, 2, 3", SC'11): rotation constants
  13,15,26,6 / 17,29,16,24 and key-schedule parity constant 0x1BD11BDA.
* JAX's key derivation: ``key(seed)`` = (seed >> 32, seed & 0xffffffff);
  ``split`` and ``random_bits`` in the "partitionable" layout, where element i
  of a shape is produced from the counter pair (hi32(i), lo32(i)); 32-bit random
  bits are the XOR of the two Threefry output words.  (The original layout,
  selectable with ``partitionable=False``, is kept for diagnosis.)
* ``uniform``: the top 23 bits are placed in the mantissa of a float in [1, 2)
  and 1 is subtracted, then scaled as ``u*(hi-lo)+lo`` and clamped below at lo.
* ``normal``: ``sqrt(2) * erfinv(u)`` with u uniform on (nextafter(-1, 0), 1),
  erfinv by the single-precision approximation of M. Giles, "Approximating the
  erfinv function" (GPU Computing Gems, 2011).  JAX's own erfinv differs from
  this one by the last-bit rounding of its log1p only, so normals agree with
  JAX's to a few ulp (well inside the fixtures' rtol 1e-4).

The reference's call sites reproduced with these primitives are cited where
they are used (``oracle/refpath.py``).
"""

from __future__ import annotations

import numpy as np

_U32 = np.uint32
_ROT = ((13, 15, 26, 6), (17, 29, 16, 24))
_PARITY = _U32(0x1BD11BDA)

# Module-level switch: the reference's JAX (>= 0.5.0) uses the partitionable layout.
PARTITIONABLE = True


def _rotl(x: np.ndarray, r: int) -> np.ndarray:
    return (x << _U32(r)) | (x >> _U32(32 - r))


def threefry2x32(k0, k1, x0, x1):
    """Threefry-2x32, 20 rounds, on uint32 arrays (broadcasting)."""
    with np.errstate(over="ignore"):
        k0 = np.asarray(k0, dtype=_U32)
        k1 = np.asarray(k1, dtype=_U32)
        ks = (k0, k1, k0 ^ k1 ^ _PARITY)
        x0 = np.asarray(x0, dtype=_U32) + ks[0]
        x1 = np.asarray(x1, dtype=_U32) + ks[1]
        for i in range(5):
            for r in _ROT[i % 2]:
                x0 = x0 + x1
                x1 = _rotl(x1, r)
                x1 = x0 ^ x1
            x0 = x0 + ks[(i + 1) % 3]
            x1 = x1 + ks[(i + 2) % 3] + _U32(i + 1)
    return x0, x1


class Key:
    """A JAX-style threefry key: a pair of uint32 words (possibly batched).

    ``data`` has shape ``batch + (2,)``.
    """

    __slots__ = ("data",)

    def __init__(self, data):
        self.data = np.asarray(data, dtype=_U32)
        assert self.data.shape[-1] == 2

    @property
    def shape(self):
        return self.data.shape[:-1]

    def __getitem__(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        return Key(self.data[idx + (slice(None),)])

    def reshape(self, *shape):
        return Key(self.data.reshape(tuple(shape) + (2,)))

    def __repr__(self):
        return f"Key({self.data.tolist()})"


def key(seed: int) -> Key:
    """``jax.random.key(seed)`` for the threefry implementation."""
    seed = int(seed)
    return Key([(seed >> 32) & 0xFFFFFFFF, seed & 0xFFFFFFFF])


def _iota_hi_lo(n: int):
    i = np.arange(n, dtype=np.uint64)
    return (i >> np.uint64(32)).astype(_U32), (i & np.uint64(0xFFFFFFFF)).astype(_U32)


def _threefry_counts(k: Key, counts: np.ndarray):
    """JAX's ``threefry_2x32(keypair, count)`` (original layout helper)."""
    counts = counts.ravel().astype(_U32)
    odd = counts.size % 2
    if odd:
        counts = np.concatenate([counts, np.zeros(1, _U32)])
    half = counts.size // 2
    y0, y1 = threefry2x32(k.data[0], k.data[1], counts[:half], counts[half:])
    out = np.concatenate([y0, y1])
    return out[:-1] if odd else out


def split(k: Key, num: int = 2) -> Key:
    """``jax.random.split`` of a single key into ``num`` keys."""
    assert k.shape == (), "split a single key"
    if PARTITIONABLE:
        hi, lo = _iota_hi_lo(num)
        b0, b1 = threefry2x32(k.data[0], k.data[1], hi, lo)
        return Key(np.stack([b0, b1], axis=-1))
    out = _threefry_counts(k, np.arange(2 * num, dtype=_U32))
    return Key(out.reshape(num, 2))


def random_bits32(k: Key, shape) -> np.ndarray:
    """``jax.random.bits`` with 32-bit width, for a single key."""
    shape = tuple(shape)
    n = int(np.prod(shape)) if shape else 1
    if PARTITIONABLE:
        if shape == ():
            hi = lo = np.zeros(1, _U32)
        else:
            hi, lo = _iota_hi_lo(n)
        b0, b1 = threefry2x32(k.data[0], k.data[1], hi, lo)
        return (b0 ^ b1).reshape(shape)
    return _threefry_counts(k, np.arange(n, dtype=_U32)).reshape(shape)


def uniform(k: Key, shape=(), minval=0.0, maxval=1.0) -> np.ndarray:
    """``jax.random.uniform`` in float32."""
    bits = random_bits32(k, shape)
    fbits = (bits >> _U32(9)) | _U32(0x3F800000)
    floats = fbits.view(np.float32) - np.float32(1.0)
    lo = np.float32(minval)
    hi = np.float32(maxval)
    span = np.float32(hi - lo)
    return np.maximum(lo, floats * span + lo).astype(np.float32)


_ERFINV_LT5 = np.array(
    [2.81022636e-08, 3.43273939e-07, -3.5233877e-06, -4.39150654e-06,
     0.00021858087, -0.00125372503, -0.00417768164, 0.246640727, 1.50140941],
    dtype=np.float32,
)
_ERFINV_GE5 = np.array(
    [-0.000200214257, 0.000100950558, 0.00134934322, -0.00367342844,
     0.00573950773, -0.0076224613, 0.00943887047, 1.00167406, 2.83297682],
    dtype=np.float32,
)


def erfinv_f32(x: np.ndarray) -> np.ndarray:
    """Giles' single-precision erfinv approximation, evaluated in float32."""
    x = np.asarray(x, dtype=np.float32)
    w = -np.log1p(-(x * x)).astype(np.float32)
    lt = w < np.float32(5.0)
    wl = (w - np.float32(2.5)).astype(np.float32)
    wg = (np.sqrt(w) - np.float32(3.0)).astype(np.float32)
    ww = np.where(lt, wl, wg).astype(np.float32)
    p = np.where(lt, _ERFINV_LT5[0], _ERFINV_GE5[0]).astype(np.float32)
    for i in range(1, 9):
        c = np.where(lt, _ERFINV_LT5[i], _ERFINV_GE5[i]).astype(np.float32)
        p = (c + p * ww).astype(np.float32)
    res = (p * x).astype(np.float32)
    return np.where(np.abs(x) == np.float32(1.0), x * np.float32(np.inf), res).astype(np.float32)


_NORMAL_LO = np.nextafter(np.float32(-1.0), np.float32(0.0), dtype=np.float32)


def normal(k: Key, shape=()) -> np.ndarray:
    """``jax.random.normal`` in float32."""
    u = uniform(k, shape, _NORMAL_LO, 1.0)
    return (np.float32(np.sqrt(2.0)) * erfinv_f32(u)).astype(np.float32)
