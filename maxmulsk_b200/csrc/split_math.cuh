// Limb arithmetic of the split-precision modes, shared by the split pre-pass
// (split.cu) and the tensor-core kernel that splits its own tiles (tc.cu), so
// that both produce the same operand bits.
//   3xTF32 : hi = rna_tf32(x), lo = rna_tf32(x - hi)
//   BF16x6 / BF16x9 : l0 = rne_bf16(x), l1 = rne_bf16(x - l0), l2 = rne_bf16(x - l0 - l1)
// x - hi and x - l0 - l1 are exact in FP32 (Sterbenz).
#pragma once

#include <cstdint>

namespace mmsk {

// Round to TF32 (10 explicit mantissa bits), nearest, ties away from zero:
// add half an ulp to the magnitude bits and clear the 13 dropped bits.
__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t b = __float_as_uint(x);
    return __uint_as_float((b + 0x1000u) & 0xFFFFE000u);
}

// Two floats to BF16, round to nearest, ties to even (the hardware
// conversion), packed as two 16-bit fields: lo in bits 0-15, hi in 16-31.
__device__ __forceinline__ uint32_t bf16x2_rn(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ float bf16_lo(uint32_t packed) { return __uint_as_float(packed << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t packed) { return __uint_as_float(packed & 0xFFFF0000u); }

// The three BF16 limbs of x0 and x1, each limb packed as a pair (x0 low).
__device__ __forceinline__ void bf16_limbs2(float x0, float x1, uint32_t& p0, uint32_t& p1, uint32_t& p2) {
    p0 = bf16x2_rn(x0, x1);
    const float r0 = x0 - bf16_lo(p0), r1 = x1 - bf16_hi(p0);
    p1 = bf16x2_rn(r0, r1);
    const float s0 = r0 - bf16_lo(p1), s1 = r1 - bf16_hi(p1);
    p2 = bf16x2_rn(s0, s1);
}

// src[0] + src[stride] + ... + src[(n - 1) stride], added in that order with
// round-to-nearest FP32 adds (the slice order of the split-K reductions); the
// loads are issued BATCH at a time so that they overlap (a batch of 64 covers
// every split in one round trip to L2).
template <int BATCH = 16>
__device__ __forceinline__ float ordered_sum(const float* __restrict__ src, size_t stride, int n) {
    float acc = __ldcs(src);
    for (int z = 1; z < n; z += BATCH) {
        float v[BATCH];
#pragma unroll
        for (int j = 0; j < BATCH; j++) v[j] = (z + j < n) ? __ldcs(src + (size_t)(z + j) * stride) : 0.0f;
#pragma unroll
        for (int j = 0; j < BATCH; j++)
            if (z + j < n) acc = __fadd_rn(acc, v[j]);
    }
    return acc;
}

}  // namespace mmsk
