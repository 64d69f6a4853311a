"""Inputs on which the split-precision products are exact in FP32, for
pinning each mode's set of limb products bit for bit (used by
tests/test_gpu_accuracy.py; the construction itself is checked on the CPU in
tests/test_oracle.py). Modes: 1 = 3xTF32, 2 = BF16x6, 3 = BF16x9."""
import numpy as np


def pinning_inputs(rng, M, K, N, mode, side, level):
    """A (M x K), B (K x N) on which every split product is exact in FP32.

    Entries are +-1, +-(1 + d1) or +-(1 + d1 + d2): BF16 limbs (1, 2^-9, 2^-17),
    TF32 limbs (1, 2^-12). Along k the entries come in pairs (k even, k + 1).
    side "a": A[:, k+1] = -(the first `level` limbs of A[:, k]) and
    B[k+1, :] = B[k, :], so in every MMA the products of the leading limbs
    cancel exactly and C = sum over pairs of (residual limbs of A) * B; side "b"
    the same with the roles of A and B swapped. All products of one limb pair
    have the same magnitude, and every partial sum fits in 24 bits, so any
    order of accumulation gives the exact value.

    Only the last MMA k-step of each 32-k accumulation chunk (16 k's for
    BF16, 8 for TF32) holds pairs; every other k is zero. Measured on B200:
    an MMA aligns its sum to its largest product, cancelling ones included,
    so an MMA of unit-size products issued after smaller terms in the same
    accumulator truncates them below about 2^-24 (BF16x9's three extra
    products, 2^-26 below the leading one, vanished that way). With the
    pairs in the chunk's last k-step, the leading limbs' MMAs meet a zero
    accumulator, and the chunk sums are added in FP32 registers."""
    tf32 = int(mode) == 1
    d = [2.0 ** -12] if tf32 else [2.0 ** -9, 2.0 ** -17]

    def full_vals(n, limbs):
        return np.float32(1.0 + sum(d[:limbs - 1])) * np.where(rng.random(n) < 0.5, -1, 1).astype(np.float32)

    def any_vals(n):
        limbs = rng.integers(1, len(d) + 2, size=n)
        v = np.ones(n, np.float64)
        for i in range(len(d)):
            v += np.where(limbs > i + 1, d[i], 0.0)
        return (v * np.where(rng.random(n) < 0.5, -1, 1)).astype(np.float32)

    limbs_needed = level + 1                      # the truncated side has residual limbs from `level` on
    A = np.empty((M, K), np.float32)
    B = np.empty((K, N), np.float32)
    half = K // 2
    if side == "a":
        x = full_vals(M * half, limbs_needed).reshape(M, half)
        lead = np.float32(1.0 + sum(d[:level - 1])) * np.sign(x)
        A[:, 0::2], A[:, 1::2] = x, -lead
        y = any_vals(half * N).reshape(half, N)
        B[0::2, :], B[1::2, :] = y, y
    else:
        y = full_vals(half * N, limbs_needed).reshape(half, N)
        lead = np.float32(1.0 + sum(d[:level - 1])) * np.sign(y)
        B[0::2, :], B[1::2, :] = y, -lead
        x = any_vals(M * half).reshape(M, half)
        A[:, 0::2], A[:, 1::2] = x, x
    kstep = 8 if tf32 else 16
    active = (np.arange(K) % 32) >= 32 - kstep
    A[:, ~active] = 0.0
    B[~active, :] = 0.0
    return A.ravel(), B.ravel()
