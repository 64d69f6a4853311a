"""Shape sets of the benchmark configurations (seeded, reproducible).

* square sweep:  M = N = K in {256, 512, 1024, 2048, 4096}
* narrow M:      M in {64, 128}, N = 512, K in {8192, 16384, 32768}, N(0, 1/K)
* grouped:       256 GEMMs, M log-uniform in [1, 512] with odd residues,
                 N in {512, 1024, 2048, 3072}, K in {512, ..., 8192} step 64
                 plus about 10% of K not a multiple of 16
* picker:        M, N, K log-uniform in [1, 16384]

The narrow-M shapes are the reference's LLM rows of its sweep
(bench/results/2026-09-13/source/bench_sweep_shapes.h:4-6); the others follow
the benchmark configurations' stated distributions.
"""
from __future__ import annotations

import numpy as np

SQUARE = [256, 512, 1024, 2048, 4096]
NARROW_M = [(m, k, 512) for m in (64, 128) for k in (8192, 16384, 32768)]


def grouped_problems(count: int = 256, seed: int = 2026) -> list[tuple[int, int, int]]:
    """(M, K, N) of the grouped batch."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m = int(np.exp(rng.uniform(0.0, np.log(512.0))))
        m = max(1, min(512, m))
        if m % 2 == 0 and rng.random() < 0.5:            # odd residues
            m = max(1, m - 1)
        n = int(rng.choice([512, 1024, 2048, 3072]))
        k = int(rng.integers(512 // 64, 8192 // 64 + 1)) * 64
        if rng.random() < 0.10:                            # not a multiple of 16
            k = max(17, k - int(rng.integers(1, 16)))
        out.append((m, k, n))
    return out


def picker_shapes(count: int, seed: int, lo: int = 1, hi: int = 16384) -> list[tuple[int, int, int]]:
    """(M, K, N), each log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    v = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=(count, 3))).astype(np.int64)
    v = np.clip(v, lo, hi)
    return [(int(a), int(b), int(c)) for a, b, c in v]
