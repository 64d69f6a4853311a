"""Generates tests/golden/multiply_scalar.json from the reference itself.

The reference ships no golden vectors (its tests fill from an unseeded
std::random_device, common/utils.hpp:13-18). This script runs the reference's
own Utils::multiply_scalar (common/utils.hpp:50-61), compiled from the
reference checkout into oracle/_ref by `make -C oracle ref`, on seeded inputs
and records, per case, the SHA-256 of the full FP32 output and 256 sampled
entries (as float32 bit patterns). It does so for two builds of the same
source: without multiply-add contraction (`sha256`, `sample_bits`) and with
it (`sha256_fma`, `sample_bits_fma`: one fused multiply-add per k step, what
the reference's own clang build emits for `sum += A*B`).

Shapes: the reference's SME correctness cases (sme/support/test_sme.cpp:28-37),
its NEON tail cases (neon/test_neon.cpp:20-40, fields M, N, K there) and one
narrow-M shape of its LLM sweep (bench/results/2026-09-13/source/bench_sweep_shapes.h:4).

Run where the reference checkout is, naming it:
    make -C oracle all ref REFERENCE_ROOT=<checkout>
    MAXMULSK_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

# (M, K, N, tag)
SME_CASES = [(16, 16, 16, "sme 16^3"), (32, 32, 32, "sme 32^3"), (64, 64, 64, "sme 64^3"),
             (67, 67, 67, "sme 67^3 all tails"), (128, 128, 128, "sme 128^3"), (20, 35, 41, "sme 20x35x41"),
             (256, 256, 256, "sme 256^3"), (512, 512, 512, "sme 512^3")]
# NEON cases are listed there as (M, N, K).
NEON_MNK = [(64, 60, 64, "neon aligned"), (128, 120, 128, "neon aligned"), (256, 240, 256, "neon aligned"),
            (67, 60, 64, "neon M tail"), (64, 65, 64, "neon N tail"), (64, 60, 65, "neon K tail"),
            (67, 65, 65, "neon all tails"), (4, 4, 4, "neon tiny"), (100, 100, 100, "neon non-aligned"),
            (128, 1100, 128, "neon N > Nc_cache")]
NARROW = [(64, 8192, 512, "llm 64x8192x512")]


def cases():
    out = list(SME_CASES)
    out += [(m, k, n, t) for (m, n, k, t) in NEON_MNK]
    out += NARROW
    return out


def main() -> None:
    if not (oracle.ref_available() and oracle.ref_fma_available()):
        oracle.build(reference_root=os.environ.get("MAXMULSK_REFERENCE_ROOT"))
    rng_pick = np.random.default_rng(20261203)
    records = []
    for i, (M, K, N, tag) in enumerate(cases()):
        seed_a, seed_b = 1000 + 2 * i, 1001 + 2 * i
        A = oracle.fill_uniform(M * K, seed_a)
        B = oracle.fill_uniform(K * N, seed_b)
        C = oracle.ref_multiply_scalar(A, B, M, K, N)
        Cf = oracle.ref_fma_multiply_scalar(A, B, M, K, N)
        idx = np.sort(rng_pick.choice(M * N, size=min(256, M * N), replace=False))
        records.append({
            "tag": tag, "M": M, "K": K, "N": N, "dist": "uniform", "seed_a": seed_a, "seed_b": seed_b,
            "sha256": hashlib.sha256(C.tobytes()).hexdigest(),
            "sample_idx": idx.tolist(),
            "sample_bits": C.ravel()[idx].view(np.uint32).tolist(),
            "sha256_fma": hashlib.sha256(Cf.tobytes()).hexdigest(),
            "sample_bits_fma": Cf.ravel()[idx].view(np.uint32).tolist(),
        })
        print(f"{tag:24s} {M}x{K}x{N}  {records[-1]['sha256'][:16]}")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "multiply_scalar.json")
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "function": "Utils::multiply_scalar (common/utils.hpp:50-61), compiled from the reference",
                   "inputs": "oracle fill_uniform(seed): SplitMix64, U[-1,1) with 24-bit resolution",
                   "cases": records}, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
