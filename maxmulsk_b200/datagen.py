"""Seeded synthetic inputs (numpy), identical bit for bit to the oracle's C
generators: SplitMix64 of (seed, index), then

* uniform : U[-1, 1) with 24-bit resolution, x = (u - 2^23) * 2^-23
* normal  : Irwin-Hall sum of 12 24-bit uniforms (exact integer sum), centred,
            rounded once to float32, times `scale` (the narrow-M inputs N(0, 1/K) use
            scale = 1/sqrt(K))
* wide    : uniform 23-bit mantissa, exponent uniform in [-20, 20], random sign

The reference fills from an unseeded std::random_device
(common/utils.hpp:13-18); these fixed-seed counterparts make every run
reproducible.
"""
from __future__ import annotations

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, idx: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx.astype(np.uint64) + np.uint64(1)) * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def _chunks(n: int, chunk: int = 1 << 22):
    for s in range(0, n, chunk):
        yield s, min(n, s + chunk)


def uniform(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    for s, e in _chunks(n):
        u = (splitmix64(seed, np.arange(s, e, dtype=np.uint64)) >> np.uint64(40)).astype(np.int64)
        out[s:e] = (u - 8388608).astype(np.float32) * np.float32(1.0 / 8388608.0)
    return out


def normal(n: int, seed: int, scale: float) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    sc = np.float32(scale)
    for s, e in _chunks(n, 1 << 20):
        base = np.arange(s, e, dtype=np.uint64) * np.uint64(12)
        acc = np.zeros(e - s, dtype=np.int64)
        for j in range(12):
            acc += (splitmix64(seed, base + np.uint64(j)) >> np.uint64(40)).astype(np.int64)
        acc -= 6 * 16777216
        z = acc.astype(np.float32) * np.float32(1.0 / 16777216.0)
        out[s:e] = z * sc
    return out


def wide(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    for s, e in _chunks(n):
        z = splitmix64(seed, np.arange(s, e, dtype=np.uint64))
        sign = ((z >> np.uint64(63)) << np.uint64(31)).astype(np.uint32)
        ex = (((z >> np.uint64(32)) & np.uint64(0xFFFF)) % np.uint64(41)).astype(np.int64) - 20
        mant = (z & np.uint64(0x7FFFFF)).astype(np.uint32)
        out[s:e] = sign | ((127 + ex).astype(np.uint32) << np.uint32(23)) | mant
    return out.view(np.float32)


def matrix(kind: str, rows: int, cols: int, seed: int, K: int | None = None) -> np.ndarray:
    """A rows x cols float32 matrix of the named distribution."""
    n = rows * cols
    if kind == "uniform":
        x = uniform(n, seed)
    elif kind == "normal":
        x = normal(n, seed, 1.0 / float(np.sqrt(K if K else cols)))
    elif kind == "wide":
        x = wide(n, seed)
    else:
        raise ValueError(kind)
    return x.reshape(rows, cols)
