// Split pre-pass: FP32 operands -> tensor-core operand planes.
//
// Replaces the reference's packers (pack_A_streaming / pack_B_streaming,
// sme/v3/sme-1x4-acc-kcout.cpp:39-193) for the split-precision path.
//   A, every mode : K-major planes [P][M][Kp].
//   B, 3xTF32     : K-major planes [P][N][Kp] (B transposed on the way: the
//                   TF32 tensor-core MMA takes B only K-major; with an
//                   N-major B operand it produces zeros).
//   B, BF16 modes : N-major planes in 128-byte column panels,
//                   [P][Np/NBE][K][NBE] with NBE = 64 BF16 elements, the GPU
//                   counterpart of the reference's 64-column B panels
//                   (packed_B[g*K_curr*64 + k*64 + c], :145-193).
// Padding is zero, so it contributes nothing, like the reference's
// zero-padded edge packs.
//
// Planes, from their definitions (finite inputs):
//   3xTF32 : hi = rna_tf32(x), lo = rna_tf32(x - hi)   (P = 2, stored as FP32
//            bit patterns with the low 13 mantissa bits clear)
//   BF16x6 / BF16x9 : l0 = rne_bf16(x), l1 = rne_bf16(x - l0),
//            l2 = rne_bf16(x - l0 - l1)                  (P = 3, stored as BF16)
// x - hi and x - l0 - l1 are exact in FP32 (Sterbenz), so hi + lo and
// l0 + l1 + l2 represent x to 2^-22 and 2^-24 relative respectively.
//
// HBM-bound: one read of each operand, P writes.
#include <cuda_runtime.h>
#include <cstdint>

#include "internal.hpp"
#include "split_math.cuh"

namespace mmsk {
namespace {

// One pass over a row-major R x Cin FP32 matrix, writing P planes of R x Cout
// (Cout >= Cin, multiple of 4; columns >= Cin are zero). Each thread handles 4
// consecutive output columns. With panel > 0 the plane is stored in column
// panels of `panel` elements: element (r, c) at ((c / panel) * R + r) * panel
// + c % panel; with panel == 0 it is stored row-major.
template <int MODE>
__global__ void __launch_bounds__(256)
split_kernel(const float* __restrict__ src, int64_t R, int64_t Cin, int64_t Cout, int64_t panel,
             void* __restrict__ planes, size_t plane_bytes) {
    const int64_t quads_per_row = Cout / 4;
    const int64_t total = R * quads_per_row;
    const bool vec = (Cin % 4 == 0) && (((uintptr_t)src & 15) == 0);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = q / quads_per_row;
        const int64_t c = (q % quads_per_row) * 4;
        float x[4];
        const float* row = src + r * Cin;
        if (vec && c + 3 < Cin) {
            float4 v = __ldcs(reinterpret_cast<const float4*>(row + c));
            x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) x[j] = (c + j < Cin) ? __ldcs(row + c + j) : 0.0f;
        }
        const size_t off = panel > 0
            ? ((size_t)(c / panel) * (size_t)R + (size_t)r) * (size_t)panel + (size_t)(c % panel)
            : (size_t)r * (size_t)Cout + (size_t)c;
        if constexpr (MODE == MAXMULSK_PREC_3XTF32) {
            float hi[4], lo[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                hi[j] = tf32_rna(x[j]);
                lo[j] = tf32_rna(x[j] - hi[j]);
            }
            float* p0 = reinterpret_cast<float*>(planes);
            float* p1 = reinterpret_cast<float*>(reinterpret_cast<char*>(planes) + plane_bytes);
            *reinterpret_cast<float4*>(p0 + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4*>(p1 + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        } else {
            uint2 l[3];
            bf16_limbs2(x[0], x[1], l[0].x, l[1].x, l[2].x);
            bf16_limbs2(x[2], x[3], l[0].y, l[1].y, l[2].y);
#pragma unroll
            for (int p = 0; p < 3; p++) {
                uint16_t* dst = reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(planes) + (size_t)p * plane_bytes);
                *reinterpret_cast<uint2*>(dst + off) = l[p];
            }
        }
    }
}

// B (K x N, row-major) -> BF16 limb planes in 128-byte column panels
// [P][Np/64][K][64] (columns >= N zero). Block unit (panel g, chunk of 64
// rows): 64 rows x 64 columns in, one contiguous 8 KB run of panel g per
// plane out. Units are numbered panel-fastest, so the blocks running at one
// time read whole rows of B, and every plane is written in long runs
// instead of 128-byte pieces one panel (K x 128 bytes) apart, which is what
// the row-major walk of split_kernel writes. A warp reads two 256-byte row
// segments and writes 256 contiguous bytes per plane; each thread takes 4
// quads, loads first.
__global__ void __launch_bounds__(256)
split_bf16_panels_kernel(const float* __restrict__ src, int64_t R, int64_t Cin, int64_t Cout,
                         void* __restrict__ planes, size_t plane_bytes) {
    constexpr int PANEL = 64, ROWS = 64, QUADS = PANEL / 4, PER = ROWS * QUADS / 256;
    const int64_t npan = Cout / PANEL;
    const int64_t units = npan * ((R + ROWS - 1) / ROWS);
    const bool vec = (Cin % 4 == 0) && (((uintptr_t)src & 15) == 0);
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int64_t g = u % npan, r0 = (u / npan) * ROWS;
        float x[PER][4];
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int idx = threadIdx.x + i * 256;
            const int64_t r = r0 + idx / QUADS, c = g * PANEL + (idx % QUADS) * 4;
            const float* row = src + r * Cin;
            if (r >= R) {
#pragma unroll
                for (int j = 0; j < 4; j++) x[i][j] = 0.0f;
            } else if (vec && c + 3 < Cin) {
                const float4 v = __ldcs(reinterpret_cast<const float4*>(row + c));
                x[i][0] = v.x; x[i][1] = v.y; x[i][2] = v.z; x[i][3] = v.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) x[i][j] = (c + j < Cin) ? __ldcs(row + c + j) : 0.0f;
            }
        }
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int idx = threadIdx.x + i * 256;
            const int64_t r = r0 + idx / QUADS;
            if (r >= R) continue;
            const size_t off = ((size_t)g * (size_t)R + (size_t)r) * PANEL + (size_t)(idx % QUADS) * 4;
            uint2 l[3];
            bf16_limbs2(x[i][0], x[i][1], l[0].x, l[1].x, l[2].x);
            bf16_limbs2(x[i][2], x[i][3], l[0].y, l[1].y, l[2].y);
#pragma unroll
            for (int p = 0; p < 3; p++) {
                uint16_t* dst = reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(planes) + (size_t)p * plane_bytes);
                *reinterpret_cast<uint2*>(dst + off) = l[p];
            }
        }
    }
}

// B (K x N, row-major) -> TF32 planes of B transposed, [P][N][Kp] with
// k >= K zero. 32 x 32 tiles through shared memory so that both the read
// (along n) and the write (along k) are coalesced.
__global__ void __launch_bounds__(256)
split_tf32_transpose_kernel(const float* __restrict__ B, int64_t K, int64_t N, int64_t Kp,
                            float* __restrict__ planes, size_t plane_bytes) {
    __shared__ float tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;     // 32 x 8
    const int64_t k0 = (int64_t)blockIdx.x * 32, n0 = (int64_t)blockIdx.y * 32;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int64_t k = k0 + ty + 8 * j, n = n0 + tx;
        tile[ty + 8 * j][tx] = (k < K && n < N) ? __ldcs(B + k * N + n) : 0.0f;
    }
    __syncthreads();
    float* hi_p = planes;
    float* lo_p = reinterpret_cast<float*>(reinterpret_cast<char*>(planes) + plane_bytes);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int64_t n = n0 + ty + 8 * j, k = k0 + tx;
        if (n < N && k < Kp) {
            const float x = tile[tx][ty + 8 * j];
            const float h = tf32_rna(x);
            hi_p[n * Kp + k] = h;
            lo_p[n * Kp + k] = tf32_rna(x - h);
        }
    }
}

inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

cudaError_t launch_tf32_transpose(const float* B, int64_t K, int64_t N, int64_t Kp, void* planes,
                                  size_t plane_bytes, cudaStream_t s) {
    if (K == 0 || N == 0) return cudaSuccess;
    dim3 grid((unsigned)((Kp + 31) / 32), (unsigned)((N + 31) / 32));
    split_tf32_transpose_kernel<<<grid, 256, 0, s>>>(B, K, N, Kp, static_cast<float*>(planes), plane_bytes);
    return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_one(const float* src, int64_t R, int64_t Cin, int64_t Cout, int64_t panel,
                       void* planes, size_t plane_bytes, cudaStream_t s) {
    const int64_t total = R * (Cout / 4);
    if (total == 0) return cudaSuccess;
    const int sms = device_sm_count();
    if (MODE != MAXMULSK_PREC_3XTF32 && panel == 64) {
        const int64_t units = (Cout / 64) * ((R + 63) / 64);
        const int64_t blocks = units < (int64_t)sms * 8 ? units : (int64_t)sms * 8;
        split_bf16_panels_kernel<<<(unsigned)blocks, 256, 0, s>>>(src, R, Cin, Cout, planes, plane_bytes);
        return cudaGetLastError();
    }
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)sms * 8;
    if (blocks > cap) blocks = cap;
    split_kernel<MODE><<<(unsigned)blocks, 256, 0, s>>>(src, R, Cin, Cout, panel, planes, plane_bytes);
    return cudaGetLastError();
}

}  // namespace

PlaneGeom plane_geom(int64_t M, int64_t K, int64_t N, int precision) {
    PlaneGeom g;
    const bool tf32 = (precision == MAXMULSK_PREC_3XTF32);
    g.P = tf32 ? 2 : 3;
    g.esize = tf32 ? 4 : 2;
    // K-major rows: a multiple of 16 bytes (TMA row stride). N-major B: a
    // whole number of 128-byte column panels.
    g.b_kmajor = tf32;
    g.Kp = (int64_t)round_up((size_t)K, (size_t)(16 / g.esize));
    g.Np = tf32 ? N : (int64_t)round_up((size_t)N, (size_t)(128 / g.esize));
    g.a_plane_bytes = round_up((size_t)M * (size_t)g.Kp * (size_t)g.esize, 1024);
    g.b_plane_bytes = tf32 ? round_up((size_t)N * (size_t)g.Kp * (size_t)g.esize, 1024)
                           : round_up((size_t)K * (size_t)g.Np * (size_t)g.esize, 1024);
    return g;
}

cudaError_t split_launch(const float* A, const float* B, int64_t M, int64_t K, int64_t N,
                         int precision, void* planes, cudaStream_t s) {
    const PlaneGeom g = plane_geom(M, K, N, precision);
    char* a_planes = static_cast<char*>(planes);
    char* b_planes = a_planes + (size_t)g.P * g.a_plane_bytes;
    cudaError_t e;
    if (precision == MAXMULSK_PREC_3XTF32) {
        e = launch_one<MAXMULSK_PREC_3XTF32>(A, M, K, g.Kp, 0, a_planes, g.a_plane_bytes, s);
        if (e != cudaSuccess) return e;
        return launch_tf32_transpose(B, K, N, g.Kp, b_planes, g.b_plane_bytes, s);
    }
    e = launch_one<MAXMULSK_PREC_BF16X6>(A, M, K, g.Kp, 0, a_planes, g.a_plane_bytes, s);
    if (e != cudaSuccess) return e;
    return launch_one<MAXMULSK_PREC_BF16X6>(B, K, N, g.Np, 128 / g.esize, b_planes, g.b_plane_bytes, s);
}

size_t split_one_bytes(int64_t R, int64_t C, int precision, bool as_b) {
    // As A: R x C is M x K. As B: R x C is K x N.
    const PlaneGeom g = as_b ? plane_geom(1, R, C, precision) : plane_geom(R, C, 1, precision);
    return (size_t)g.P * (as_b ? g.b_plane_bytes : g.a_plane_bytes);
}

cudaError_t split_one(const float* X, int64_t R, int64_t C, int precision, bool as_b, void* out,
                      cudaStream_t s) {
    const PlaneGeom g = as_b ? plane_geom(1, R, C, precision) : plane_geom(R, C, 1, precision);
    if (precision == MAXMULSK_PREC_3XTF32) {
        if (as_b) return launch_tf32_transpose(X, R, C, g.Kp, out, g.b_plane_bytes, s);
        return launch_one<MAXMULSK_PREC_3XTF32>(X, R, C, g.Kp, 0, out, g.a_plane_bytes, s);
    }
    if (as_b) return launch_one<MAXMULSK_PREC_BF16X6>(X, R, C, g.Np, 128 / g.esize, out, g.b_plane_bytes, s);
    return launch_one<MAXMULSK_PREC_BF16X6>(X, R, C, g.Kp, 0, out, g.a_plane_bytes, s);
}

}  // namespace mmsk
