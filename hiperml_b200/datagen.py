"""Seeded synthetic inputs for the skinny SGEMM/SGEMV workloads.

The generator is counter based (SplitMix64 output function), so any element
of any buffer can be produced independently and the device generator
(``hml_fill_random`` in the native library) yields the same values:

* ``key   = mix(mix(seed) ^ (stream * 0xD6E8FEB86659FD93))``
* ``z_i   = mix(key + (i + 1) * 0x9E3779B97F4A7C15)`` for storage index ``i``
* ``UNIFORM``   ``2 * (z_i >> 40) * 2**-24 - 1``      in [-1, 1), exact in FP32
* ``NORMAL``    Box-Muller on ``u1 = ((z>>40)+1)*2**-24``, ``u2 = ((z>>16)&0xFFFFFF)*2**-24``,
  evaluated in double then rounded to FP32 (host and device may differ by one
  FP32 ulp on rare inputs because their libm differ)
* ``LOGUNIFORM`` magnitude ``10**(6*u - 3)`` (1e-3 .. 1e3), sign from bit 39,
  evaluated in double then rounded to FP32

``mix`` is the SplitMix64 finaliser.  Values depend on the storage index, so
a column-major and a row-major buffer of the same logical matrix are filled
by indexing the storage, and logical equality is obtained by transposition.
"""
from __future__ import annotations

import numpy as np

UNIFORM = 0
NORMAL = 1
LOGUNIFORM = 2

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_STREAM = 0xD6E8FEB86659FD93
_MASK = (1 << 64) - 1


def _mix_int(z: int) -> int:
    z &= _MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
    return z ^ (z >> 31)


def stream_key(seed: int, stream: int) -> int:
    return _mix_int(_mix_int(seed) ^ ((stream * _STREAM) & _MASK))


def _mix(z):
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def raw64(n: int, seed: int, stream: int, start: int = 0) -> np.ndarray:
    key = np.uint64(stream_key(seed, stream))
    idx = np.arange(start + 1, start + n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _mix(key + idx * _GOLDEN)


def fill(n: int, seed: int, stream: int, dist: int = UNIFORM,
         chunk: int = 1 << 24) -> np.ndarray:
    """``n`` FP32 values of distribution ``dist`` for (seed, stream)."""
    out = np.empty(n, np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        z = raw64(e - s, seed, stream, s)
        hi24 = (z >> np.uint64(40)).astype(np.float64)
        if dist == UNIFORM:
            out[s:e] = (2.0 * (hi24 * 2.0 ** -24) - 1.0).astype(np.float32)
        elif dist == NORMAL:
            u1 = (hi24 + 1.0) * 2.0 ** -24
            u2 = ((z >> np.uint64(16)) & np.uint64(0xFFFFFF)).astype(np.float64) * 2.0 ** -24
            out[s:e] = (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)).astype(np.float32)
        elif dist == LOGUNIFORM:
            mag = np.power(10.0, 6.0 * (hi24 * 2.0 ** -24) - 3.0)
            sign = np.where(((z >> np.uint64(39)) & np.uint64(1)) == 1, -1.0, 1.0)
            out[s:e] = (sign * mag).astype(np.float32)
        else:
            raise ValueError(f"unknown distribution {dist}")
    return out


def matrix(rows: int, cols: int, seed: int, stream: int, dist: int = UNIFORM,
           order: str = "F") -> np.ndarray:
    """A rows x cols FP32 matrix whose storage (column-major for ``order='F'``,
    row-major for ``'C'``) is filled in index order."""
    flat = fill(rows * cols, seed, stream, dist)
    if order == "F":
        return flat.reshape(cols, rows).T
    return flat.reshape(rows, cols)
