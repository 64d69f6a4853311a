"""The oracle itself, pinned to the reference (CPU only).

The oracle restates Utils::multiply_scalar (common/utils.hpp:50-61); these
tests pin it bit for bit to the reference's own function, both through the
committed golden fixtures and, where the reference checkout was compiled
here (oracle/_ref), live on fresh inputs.
"""
import hashlib
from fractions import Fraction

import numpy as np
import pytest

from maxmulsk_b200 import datagen


def test_golden_fixtures_pin_oracle(oracle_mod, golden_cases):
    assert len(golden_cases) >= 19
    for c in golden_cases:
        M, K, N = c["M"], c["K"], c["N"]
        A = oracle_mod.fill_uniform(M * K, c["seed_a"])
        B = oracle_mod.fill_uniform(K * N, c["seed_b"])
        C = oracle_mod.sgemm_scalar(A, B, M, K, N)
        assert hashlib.sha256(C.tobytes()).hexdigest() == c["sha256"], c["tag"]
        got = C.ravel()[np.array(c["sample_idx"])].view(np.uint32)
        assert got.tolist() == c["sample_bits"], c["tag"]
        # The contracted build is one FMA chain per output: the panel oracle
        # with a single panel and fused steps.
        Cf = oracle_mod.sgemm_panels(A, B, M, K, N, kc=0, fma=True)
        assert hashlib.sha256(Cf.tobytes()).hexdigest() == c["sha256_fma"], c["tag"]


@pytest.mark.skipif("not __import__('oracle').ref_available()")
def test_oracle_bit_exact_vs_reference_live(oracle_mod):
    rng = np.random.default_rng(7)
    for _ in range(12):
        M, K, N = (int(x) for x in rng.integers(1, 90, size=3))
        A = oracle_mod.fill_uniform(M * K, int(rng.integers(1 << 30)))
        B = oracle_mod.fill_uniform(K * N, int(rng.integers(1 << 30)))
        ours = oracle_mod.sgemm_scalar(A, B, M, K, N)
        theirs = oracle_mod.ref_multiply_scalar(A, B, M, K, N)
        assert np.array_equal(ours.view(np.uint32), theirs.view(np.uint32))


@pytest.mark.skipif("not __import__('oracle').ref_fma_available()")
def test_fma_oracle_bit_exact_vs_contracted_reference(oracle_mod):
    rng = np.random.default_rng(8)
    for _ in range(12):
        M, K, N = (int(x) for x in rng.integers(1, 90, size=3))
        A = oracle_mod.fill_uniform(M * K, int(rng.integers(1 << 30)))
        B = oracle_mod.fill_uniform(K * N, int(rng.integers(1 << 30)))
        ours = oracle_mod.sgemm_panels(A, B, M, K, N, kc=0, fma=True)
        theirs = oracle_mod.ref_fma_multiply_scalar(A, B, M, K, N)
        assert np.array_equal(ours.view(np.uint32), theirs.view(np.uint32))


@pytest.mark.skipif("not __import__('oracle').ref_available()")
def test_check_correctness_matches_reference(oracle_mod):
    x = oracle_mod.fill_uniform(1000, 3)
    y = x.copy()
    y[17] += 2e-3
    y[400] -= 5e-4
    bad, md = oracle_mod.check_correctness(x, y, 1e-3)
    assert bad == 1 and md > 1e-3
    assert oracle_mod.ref_check_correctness(x, y, 1e-3) is False
    assert oracle_mod.ref_check_correctness(x, x, 1e-3) is True


def test_numpy_generators_match_oracle(oracle_mod):
    for seed in (0, 1, 12345):
        n = 10007
        assert np.array_equal(datagen.uniform(n, seed).view(np.uint32), oracle_mod.fill_uniform(n, seed).view(np.uint32))
        sc = 1.0 / np.sqrt(8192.0)
        assert np.array_equal(datagen.normal(n, seed, sc).view(np.uint32),
                              oracle_mod.fill_normal(n, seed, sc).view(np.uint32))
        assert np.array_equal(datagen.wide(n, seed).view(np.uint32), oracle_mod.fill_wide(n, seed).view(np.uint32))


def test_generator_distributions(oracle_mod):
    u = oracle_mod.fill_uniform(1 << 16, 5)
    assert u.min() >= -1.0 and u.max() < 1.0 and abs(u.mean()) < 0.02
    z = oracle_mod.fill_normal(1 << 16, 5, 1.0)
    assert abs(z.std() - 1.0) < 0.02 and abs(z.mean()) < 0.02
    w = oracle_mod.fill_wide(1 << 16, 5)
    e = np.frexp(np.abs(w))[1] - 1
    assert e.min() == -20 and e.max() == 20
    assert (w < 0).mean() > 0.45


def test_panels_without_fma_equal_scalar(oracle_mod):
    M, K, N = 23, 77, 31
    A = oracle_mod.fill_uniform(M * K, 1)
    B = oracle_mod.fill_uniform(K * N, 2)
    s = oracle_mod.sgemm_scalar(A, B, M, K, N)
    p = oracle_mod.sgemm_panels(A, B, M, K, N, kc=0, fma=False)
    assert np.array_equal(s.view(np.uint32), p.view(np.uint32))


def _round_f32(fr: Fraction) -> np.float32:
    """Correct rounding of an exact rational to float32 (ties to even)."""
    f = np.float32(float(fr))
    cands = [np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))]
    return min(cands, key=lambda c: (abs(Fraction(float(c)) - fr), int(np.float32(c).view(np.uint32)) & 1))


def test_panels_order_by_hand(oracle_mod):
    # C = ((p0 + p1) + p2), each panel a chain of fused multiply-adds from +0.
    M, K, N, kc = 2, 10, 3, 4
    A = oracle_mod.fill_uniform(M * K, 11)
    B = oracle_mod.fill_uniform(K * N, 12)
    got = oracle_mod.sgemm_panels(A, B, M, K, N, kc=kc, fma=True)
    A2, B2 = A.reshape(M, K), B.reshape(K, N)
    for i in range(M):
        for j in range(N):
            c = None
            for k0 in range(0, K, kc):
                p = np.float32(0)
                for k in range(k0, min(K, k0 + kc)):
                    p = _round_f32(Fraction(float(A2[i, k])) * Fraction(float(B2[k, j])) + Fraction(float(p)))
                c = p if c is None else np.float32(c + p)
            assert got[i, j] == c


def test_dgemm_matches_numpy(oracle_mod):
    M, K, N = 37, 129, 53
    A = oracle_mod.fill_uniform(M * K, 21)
    B = oracle_mod.fill_uniform(K * N, 22)
    C64 = oracle_mod.dgemm(A, B, M, K, N, threads=3)
    ref = A.reshape(M, K).astype(np.float64) @ B.reshape(K, N).astype(np.float64)
    assert np.max(np.abs(C64 - ref)) < 1e-12
    rows = oracle_mod.dgemm_rows(A, B, K, N, [0, 5, 36])
    assert np.array_equal(rows, C64[[0, 5, 36]])


def test_error_measures(oracle_mod):
    M, K, N = 16, 32, 8
    A = oracle_mod.fill_uniform(M * K, 31)
    B = oracle_mod.fill_uniform(K * N, 32)
    C64 = oracle_mod.dgemm(A, B, M, K, N)
    exact = oracle_mod.errors(C64.astype(np.float32), C64, A, B, M, K, N)
    assert exact["normwise"] < 1e-7 and exact["rel_frob"] < 1e-7
    C = C64.astype(np.float32)
    C[3, 4] += 1.0
    e = oracle_mod.errors(C, C64, A, B, M, K, N)
    assert abs(e["max_abs"] - 1.0) < 1e-6
    na = np.linalg.norm(A.astype(np.float64))
    nb = np.linalg.norm(B.astype(np.float64))
    assert abs(e["normwise"] - 1.0 / (na * nb)) < 1e-6 / (na * nb)


def test_split_tf32_definition(oracle_mod):
    x = np.concatenate([oracle_mod.fill_uniform(4096, 41), oracle_mod.fill_wide(4096, 42)])
    hi, lo = oracle_mod.split_tf32(x)
    assert np.all((hi.view(np.uint32) & 0x1FFF) == 0)
    assert np.all((lo.view(np.uint32) & 0x1FFF) == 0)
    r = np.abs(x.astype(np.float64) - hi.astype(np.float64) - lo.astype(np.float64))
    assert np.all(r <= 2.0 ** -22 * np.abs(x.astype(np.float64)) + 1e-45)
    # round to nearest, ties away: |x - hi| <= half an ulp of the 11-bit significand
    assert np.all(np.abs(x.astype(np.float64) - hi) <= 2.0 ** -11 * np.abs(x.astype(np.float64)))


def test_split_bf16_definition(oracle_mod):
    x = np.concatenate([oracle_mod.fill_uniform(4096, 43), oracle_mod.fill_wide(4096, 44)])
    l0, l1, l2 = oracle_mod.split_bf16(x)
    for limb in (l0, l1, l2):
        assert np.all((limb.view(np.uint32) & 0xFFFF) == 0)
    r = np.abs(x.astype(np.float64) - l0 - l1.astype(np.float64) - l2.astype(np.float64))
    assert np.all(r <= 2.0 ** -24 * np.abs(x.astype(np.float64)))


def test_split_exact_products(oracle_mod):
    M, K, N = 9, 40, 11
    A = oracle_mod.fill_uniform(M * K, 51)
    B = oracle_mod.fill_uniform(K * N, 52)
    C64 = oracle_mod.dgemm(A, B, M, K, N)
    for mode, tol in ((1, 2e-6), (2, 2e-7), (3, 2e-7)):
        C = oracle_mod.sgemm_split_exact(A, B, M, K, N, mode)
        e = oracle_mod.errors(C, C64, A, B, M, K, N)
        assert e["normwise"] < tol, (mode, e)


# --------------------------------------------------------------------------- pinning inputs
def _kept_pairs(mode):
    if mode == 1:
        return [(0, 0), (0, 1), (1, 0)]
    if mode == 2:
        return [(i, j) for i in range(3) for j in range(3) if i + j <= 2]
    return [(i, j) for i in range(3) for j in range(3)]


@pytest.mark.parametrize("mode,side,level", [(1, "a", 1), (1, "b", 1), (2, "a", 1), (2, "a", 2), (2, "b", 2),
                                             (3, "a", 1), (3, "b", 2)])
def test_pinning_inputs_are_exact_in_fp32(oracle_mod, mode, side, level):
    # The GPU pins compare the tensor-core result with the exact split product
    # bit for bit; that is sound only if, in the order the hardware may add
    # them, every partial sum is exact in FP32. One MMA covers one limb pair
    # over an aligned block of k's, so the two halves of a k pair (whose
    # leading-limb products cancel) meet inside one MMA. Here: each k pair of
    # each kept limb pair summed first (exactly), then those sums added in FP32
    # in k order, in reverse, and limb pair by limb pair -- all equal the
    # FP64-accumulated exact split product.
    from pinning import pinning_inputs
    rng = np.random.default_rng(mode * 100 + level)
    M, K, N = 9, 64, 11
    A, B = pinning_inputs(rng, M, K, N, mode, side, level)
    want = oracle_mod.sgemm_split_exact(A, B, M, K, N, mode)
    if mode == 1:
        la, lb = oracle_mod.split_tf32(A), oracle_mod.split_tf32(B)
    else:
        la, lb = oracle_mod.split_bf16(A), oracle_mod.split_bf16(B)
    la = [x.reshape(M, K) for x in la]
    lb = [x.reshape(K, N) for x in lb]
    terms = np.stack([la[i][:, :, None] * lb[j][None, :, :] for (i, j) in _kept_pairs(mode)])  # (P, M, K, N)
    assert terms.dtype == np.float32
    pairs = terms[:, :, 0::2, :] + terms[:, :, 1::2, :]
    assert np.array_equal(pairs.astype(np.float64),
                          terms[:, :, 0::2, :].astype(np.float64) + terms[:, :, 1::2, :].astype(np.float64))
    P, H = pairs.shape[0], pairs.shape[2]
    orders = [[(p, h) for h in range(H) for p in range(P)],
              [(p, h) for p in reversed(range(P)) for h in reversed(range(H))],
              [(p, h) for p in range(P) for h in range(H)]]
    for order in orders:
        acc = np.zeros((M, N), np.float32)
        for p, h in order:
            acc = acc + pairs[p, :, h, :]
        assert np.array_equal(acc, want)


def test_pinning_inputs_separate_the_modes(oracle_mod):
    # On the pinning inputs the modes' exact products differ from one another
    # and from the full product, so a kernel that computed a different set of
    # limb products cannot match the pins.
    from pinning import pinning_inputs
    rng = np.random.default_rng(7)
    M, K, N = 16, 32, 24
    for side in ("a", "b"):
        for level in (1, 2):
            A, B = pinning_inputs(rng, M, K, N, 2, side, level)
            assert not np.array_equal(oracle_mod.sgemm_split_exact(A, B, M, K, N, 2),
                                      oracle_mod.sgemm_split_exact(A, B, M, K, N, 3)), (side, level)
        A, B = pinning_inputs(rng, M, K, N, 1, side, 1)
        tf = oracle_mod.sgemm_split_exact(A, B, M, K, N, 1)
        full = oracle_mod.dgemm(A, B, M, K, N).astype(np.float32)
        assert not np.array_equal(tf, full), side
