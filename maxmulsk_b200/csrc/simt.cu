// FP32 SIMT GEMM for sm_100a: C = A*B, row-major, on the CUDA cores.
//
// Replaces the reference's blocked SME driver (sme/v3/sme-1x4-acc-kcout.cpp:427-567)
// as the FP32-accurate path. The SME packers (pack_A_streaming :39-136 with
// its ZA transpose, pack_B_streaming :145-193) become shared-memory staging:
// A is stored k-major (transposed on the way in, like the ZA transpose), B
// row-major; both double-buffered, fed by 128-bit global loads. The 16x64 ZA
// micro-tile becomes a CTA tile of tile_m x tile_n with an 8x8 (or 4x4)
// register tile per thread.
//
// Arithmetic: every output is ONE sequential chain over k in increasing order
// (a fused multiply-add per step, or multiply-then-add in the SCALAR variant,
// the arithmetic of Utils::multiply_scalar, common/utils.hpp:50-61). With
// split_k > 1 each K slice is such a chain and the slices are summed in slice
// order, first slice first: C = ((p0 + p1) + p2) + ..., the order in which
// the reference's v3 adds its outer-Kc panels (first_k store, then
// store_za_add; sme/v3/sme-1x4-acc-kcout.cpp:464-471, 530-558). The result is
// therefore deterministic and reproducible bit for bit by a scalar loop.
//
// Edges (the reference's scratch-tile path, :539-558) are predicated loads
// that read zero outside the matrix and predicated stores; C outside the
// matrix is never touched.
#include <cuda.h>
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "internal.hpp"
#include "phase.hpp"
#include "runtime.hpp"
#include "split_math.cuh"

namespace mmsk {
namespace {

constexpr int kThreads = 256;
constexpr int kBK = 16;

template <bool FUSED>
__device__ __forceinline__ float mac(float a, float b, float c) {
    if constexpr (FUSED) return __fmaf_rn(a, b, c);
    else return __fadd_rn(c, __fmul_rn(a, b));
}

// Shared-memory stages of one CTA.
//
// A is stored k-major: As[k][m ^ swz(k)]. A warp's transposing stores write
// 8 rows for each of the k's kq, kq+4, kq+8, kq+12 of its float4 loads; with
// rows of BM + 4 floats, k and k + 8 fall on the same banks, so rows of k >= 8
// are stored with bit 3 of the row index flipped. Groups of four rows stay
// contiguous and 16-byte aligned for the float4 reads of the product loop.
template <int BM, int BN>
struct SimtSmem {
    float As[2][kBK][BM + 4];                       // k-major A, padded rows, swizzled
    float Bs[2][kBK][BN];
    int last;
};

// The end of one tile: without a K split the sums go to C; with one, this
// slice's partial tile is written and, unless a separate reduction kernel
// follows, the last CTA of the tile to arrive sums all slices in slice order
// (C = ((p0 + p1) + p2) + ...). acc[i][4 g + j] is the output at row
// out_row(i), column out_col(g) + j. `last_flag` is a shared-memory word.
template <int TM, int GN, class RowFn, class ColFn>
__device__ __forceinline__ void simt_epilogue(const SimtArgs& p, float (&acc)[TM][4 * GN], RowFn out_row,
                                              ColFn out_col, bool VEC, int z, unsigned tile, int& last_flag) {
    const int64_t M = p.M, N = p.N;
    const int tid = threadIdx.x;
    if (p.splits <= 1) {
#pragma unroll
        for (int i = 0; i < TM; i++) {
            const int64_t r = out_row(i);
            if (r >= M) continue;
#pragma unroll
            for (int g = 0; g < GN; g++) {
                const int64_t c = out_col(g);
                float* dst = p.C + r * N + c;
                if (VEC && c + 3 < N) {
                    *reinterpret_cast<float4*>(dst) =
                        make_float4(acc[i][g * 4 + 0], acc[i][g * 4 + 1], acc[i][g * 4 + 2], acc[i][g * 4 + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (c + j < N) dst[j] = acc[i][g * 4 + j];
                }
            }
        }
        return;
    }

    // Split-K: write this slice's partial tile, then the last CTA of the tile
    // to arrive sums all slices in slice order.
    const size_t MN = (size_t)M * (size_t)N;
    float* mine = p.partial + (size_t)z * MN;
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int64_t r = out_row(i);
        if (r >= M) continue;
#pragma unroll
        for (int g = 0; g < GN; g++) {
            const int64_t c = out_col(g);
            if (VEC && c + 3 < N) {
                __stcg(reinterpret_cast<float4*>(mine + r * N + c),
                       make_float4(acc[i][g * 4 + 0], acc[i][g * 4 + 1], acc[i][g * 4 + 2], acc[i][g * 4 + 3]));
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (c + j < N) __stcg(mine + r * N + c + j, acc[i][g * 4 + j]);
            }
        }
    }
    if (p.reduce_after) return;                      // summed by simt_splitk_reduce_kernel
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        unsigned prev = atomicAdd(&p.counters[tile], 1u);
        last_flag = (prev == (unsigned)(p.splits - 1));
    }
    __syncthreads();
    const int last = last_flag;
    __syncthreads();                                 // the flag may be rewritten by the next tile
    if (!last) return;
    __threadfence();
    // Each output: slice 0, then every later slice added in slice order; four
    // adjacent columns at a time with 128-bit loads where rows allow.
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int64_t r = out_row(i);
        if (r >= M) continue;
#pragma unroll
        for (int g = 0; g < GN; g++) {
            const int64_t c = out_col(g);
            const size_t off = (size_t)r * N + c;
            if (VEC && c + 3 < N) {
                float4 s4 = __ldcg(reinterpret_cast<const float4*>(p.partial + off));
                for (int q = 1; q < p.splits; q++) {
                    const float4 t = __ldcg(reinterpret_cast<const float4*>(p.partial + (size_t)q * MN + off));
                    s4.x = __fadd_rn(s4.x, t.x); s4.y = __fadd_rn(s4.y, t.y);
                    s4.z = __fadd_rn(s4.z, t.z); s4.w = __fadd_rn(s4.w, t.w);
                }
                *reinterpret_cast<float4*>(p.C + off) = s4;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if (c + j >= N) continue;
                    float v = __ldcg(p.partial + off + j);
                    for (int q = 1; q < p.splits; q++) v = __fadd_rn(v, __ldcg(p.partial + (size_t)q * MN + off + j));
                    p.C[off + j] = v;
                }
            }
        }
    }
    if (tid == 0) p.counters[tile] = 0u;   // leave the counter ready for the next call
}

// One CTA computes the BM x BN tile at (m0, n0) of K slice z; `tile` numbers
// the tile for the split-K arrival counters. VM selects 128-bit loads and
// stores: 0 never, 1 always (both fixed at compile time), 2 at run time by
// `vec_rt` (one body for problems of either kind, as in grouped launches).
template <int BM, int BN, bool FUSED, int VM>
__device__ __forceinline__ void simt_tile(const SimtArgs& p, int64_t m0, int64_t n0, int z, unsigned tile,
                                          SimtSmem<BM, BN>& sm, bool vec_rt = false) {
    const bool VEC = (VM == 2) ? vec_rt : (VM == 1);
    constexpr int TM = BM / 16, TN = BN / 16;       // per-thread outputs
    constexpr int GM = TM / 4, GN = TN / 4;         // 4-wide groups per thread
    constexpr int A_F4 = BM * kBK / 4 / kThreads;   // float4 loads per thread
    constexpr int B_F4 = BN * kBK / 4 / kThreads;
    auto& As = sm.As;
    auto& Bs = sm.Bs;

    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int64_t kbeg = (int64_t)z * p.kchunk;
    const int64_t kend = min(p.K, kbeg + p.kchunk);
    const int64_t M = p.M, N = p.N, K = p.K;
    const float* __restrict__ A = p.A;
    const float* __restrict__ B = p.B;

    float4 ra[A_F4], rb[B_F4];

    auto load_tile = [&](int64_t k0) {
#pragma unroll
        for (int j = 0; j < A_F4; j++) {
            const int f = tid + j * kThreads;
            const int row = f / (kBK / 4);
            const int kq = (f % (kBK / 4)) * 4;
            const int64_t gm = m0 + row, gk = k0 + kq;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gm < M) {
                const float* src = A + gm * K + gk;
                if (VEC) {
                    if (gk < kend) v = __ldg(reinterpret_cast<const float4*>(src));
                } else {
                    if (gk + 0 < kend) v.x = __ldg(src + 0);
                    if (gk + 1 < kend) v.y = __ldg(src + 1);
                    if (gk + 2 < kend) v.z = __ldg(src + 2);
                    if (gk + 3 < kend) v.w = __ldg(src + 3);
                }
            }
            ra[j] = v;
        }
#pragma unroll
        for (int j = 0; j < B_F4; j++) {
            const int f = tid + j * kThreads;
            const int kr = f / (BN / 4);
            const int nq = (f % (BN / 4)) * 4;
            const int64_t gk = k0 + kr, gn = n0 + nq;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gk < kend) {
                const float* src = B + gk * N + gn;
                if (VEC) {
                    if (gn < N) v = __ldg(reinterpret_cast<const float4*>(src));
                } else {
                    if (gn + 0 < N) v.x = __ldg(src + 0);
                    if (gn + 1 < N) v.y = __ldg(src + 1);
                    if (gn + 2 < N) v.z = __ldg(src + 2);
                    if (gn + 3 < N) v.w = __ldg(src + 3);
                }
            }
            rb[j] = v;
        }
    };
    auto store_tile = [&](int buf) {
#pragma unroll
        for (int j = 0; j < A_F4; j++) {
            const int f = tid + j * kThreads;
            const int row = f / (kBK / 4);
            const int kq = (f % (kBK / 4)) * 4;
            const int srow = row ^ (kq & 8);
            As[buf][kq + 0][srow] = ra[j].x;
            As[buf][kq + 1][srow] = ra[j].y;
            As[buf][kq + 2][srow] = ra[j].z;
            As[buf][kq + 3][srow] = ra[j].w;
        }
#pragma unroll
        for (int j = 0; j < B_F4; j++) {
            const int f = tid + j * kThreads;
            const int kr = f / (BN / 4);
            const int nq = (f % (BN / 4)) * 4;
            *reinterpret_cast<float4*>(&Bs[buf][kr][nq]) = rb[j];
        }
    };

    float acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = 0.f;

    const int64_t ntiles = (kend - kbeg + kBK - 1) / kBK;
    if (ntiles > 0) {
        load_tile(kbeg);
        store_tile(0);
        __syncthreads();
        for (int64_t t = 0; t < ntiles; t++) {
            const int buf = (int)(t & 1);
            if (t + 1 < ntiles) load_tile(kbeg + (t + 1) * kBK);
            // Fragments of step k + 1 are read from shared memory while the
            // products of step k run (two register sets, fully unrolled).
            float a[2][TM], b[2][TN];
            auto load_frag = [&](int set, int k) {
#pragma unroll
                for (int g = 0; g < GM; g++) {
                    float4 v = *reinterpret_cast<const float4*>(&As[buf][k][(g * 64 + ty * 4) ^ (k & 8)]);
                    a[set][g * 4 + 0] = v.x; a[set][g * 4 + 1] = v.y; a[set][g * 4 + 2] = v.z; a[set][g * 4 + 3] = v.w;
                }
#pragma unroll
                for (int g = 0; g < GN; g++) {
                    float4 v = *reinterpret_cast<const float4*>(&Bs[buf][k][g * 64 + tx * 4]);
                    b[set][g * 4 + 0] = v.x; b[set][g * 4 + 1] = v.y; b[set][g * 4 + 2] = v.z; b[set][g * 4 + 3] = v.w;
                }
            };
            load_frag(0, 0);
#pragma unroll
            for (int k = 0; k < kBK; k++) {
                if (k + 1 < kBK) load_frag((k + 1) & 1, k + 1);
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++) acc[i][j] = mac<FUSED>(a[k & 1][i], b[k & 1][j], acc[i][j]);
            }
            if (t + 1 < ntiles) store_tile(buf ^ 1);
            __syncthreads();
        }
    }

    // Steps past kend multiply by a zero operand. The product is +-0 and adding
    // it leaves the chain unchanged (the chain never holds -0: it starts at +0
    // and an exact zero sum rounds to +0), so the padded steps keep the result
    // identical to a chain over [kbeg, kend) alone.

    auto out_row = [&](int i) { return m0 + (i / 4) * 64 + ty * 4 + (i % 4); };
    auto out_col = [&](int g) { return n0 + g * 64 + tx * 4; };
    simt_epilogue<TM, GN>(p, acc, out_row, out_col, VEC, z, tile, sm.last);
}

template <int BM, int BN, bool FUSED, bool VEC>
__global__ void __launch_bounds__(kThreads, 2)
sgemm_simt_kernel(SimtArgs p) {
    __shared__ __align__(16) SimtSmem<BM, BN> sm;
    simt_tile<BM, BN, FUSED, VEC ? 1 : 0>(p, (int64_t)blockIdx.y * BM, (int64_t)blockIdx.x * BN, blockIdx.z,
                                          blockIdx.y * gridDim.x + blockIdx.x, sm);
}

// ---------------------------------------------------------------------------
// 128 x 128 tiles on a cp.async pipeline (the plan's 128 x 128 FP32 tile).
//
// 128 threads (four warps of 64 x 64), each owning 8 x 16 outputs: rows
// wm*64 + lm + 8i (i < 8), columns wn*64 + 4 ln + 16 j + {0..3} (j < 4), with
// lane = 4 lm + ln. Two CTAs per SM. Tiles of A (128 rows x 32 k, row-major,
// rows padded to 36 floats) and B (32 k x 128 columns) arrive by cp.async
// (16-byte copies where K and N are multiples of 4 and A, B, C are 16-byte
// aligned; 4-byte copies otherwise) into a ring of three stages, so no thread
// stages operands through registers or transposes them. Per four k's a
// thread reads its 8 rows of A as 128-bit loads (4 k's each; a warp's eight
// rows fall on eight bank groups) and, per k, 16 values of B (four 128-bit
// loads, 64 contiguous bytes per warp): 512 multiply-adds per 24 shared loads.
//
// Arithmetic: as in the kernel above, every output is one chain over k in
// increasing order (the stage loop, then four k's per A load, in order), so
// C is the same bit for bit; copies outside the matrix fill zeros.
// ---------------------------------------------------------------------------
namespace cpk {
constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3;
constexpr int AST = BK + 4;                    // A row stride (floats): eight rows on eight bank groups
constexpr int A_FLOATS = BM * AST;
constexpr int B_FLOATS = BK * BN;
constexpr int STAGE_FLOATS = A_FLOATS + B_FLOATS;
constexpr int SMEM = STAGES * STAGE_FLOATS * 4;
// LT = outputs per thread along N: 16 (128 threads, warps of 64 x 64) or 8
// (256 threads, warps of 64 x 32); eight rows per thread either way.
template <int LT> struct Shape {
    static constexpr int THREADS = LT == 16 ? 128 : 256;
    static constexpr int WARPS_N = LT == 16 ? 2 : 4;
    static constexpr int WN = BN / WARPS_N;    // warp tile columns
};
}  // namespace cpk

__device__ __forceinline__ void cp_async_16(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_4(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <bool FUSED, bool VEC, int LT>
__global__ void __launch_bounds__(cpk::Shape<LT>::THREADS, 2)
sgemm_simt_cp_kernel(SimtArgs p) {
    using namespace cpk;
    constexpr int THREADS = Shape<LT>::THREADS, WARPS_N = Shape<LT>::WARPS_N, WN = Shape<LT>::WN;
    constexpr int GN = LT / 4;                 // float4 groups per thread row
    extern __shared__ __align__(16) float smem[];
    __shared__ int last_flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp / WARPS_N, wn = warp % WARPS_N;
    const int lm = lane >> 2, ln = lane & 3;
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    const int z = blockIdx.z;
    const int64_t M = p.M, N = p.N, K = p.K;
    const int64_t kbeg = (int64_t)z * p.kchunk;
    const int64_t kend = min(K, kbeg + p.kchunk);
    const int64_t ntiles = (kend - kbeg + BK - 1) / BK;
    const float* __restrict__ A = p.A;
    const float* __restrict__ B = p.B;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);

    // Stage `buf` <- A[m0.., k0..k0+BK), B[k0..k0+BK, n0..); zeros outside the
    // matrix and past kend (a copy of 0 source bytes reads nothing; its source
    // address is kept inside the operand anyway).
    auto load_stage = [&](int buf, int64_t k0) {
        const uint32_t a_s = sbase + (uint32_t)(buf * STAGE_FLOATS) * 4u;
        const uint32_t b_s = a_s + (uint32_t)A_FLOATS * 4u;
        if constexpr (VEC) {
#pragma unroll
            for (int j = 0; j < BM * BK / 4 / THREADS; j++) {       // 16-byte chunks of A
                const int c = tid + j * THREADS;
                const int row = c >> 3, ch = c & 7;
                const int64_t gm = m0 + row, gk = k0 + ch * 4;
                const bool ok = gm < M && gk < kend;
                cp_async_16(a_s + (uint32_t)(row * AST + ch * 4) * 4u, ok ? A + gm * K + gk : A, ok ? 16 : 0);
            }
#pragma unroll
            for (int j = 0; j < BK * BN / 4 / THREADS; j++) {       // 16-byte chunks of B
                const int c = tid + j * THREADS;
                const int row = c >> 5, ch = c & 31;
                const int64_t gk = k0 + row, gn = n0 + ch * 4;
                const bool ok = gk < kend && gn < N;
                cp_async_16(b_s + (uint32_t)(row * BN + ch * 4) * 4u, ok ? B + gk * N + gn : B, ok ? 16 : 0);
            }
        } else {
#pragma unroll 8
            for (int j = 0; j < BM * BK / THREADS; j++) {           // elements of A
                const int c = tid + j * THREADS;
                const int row = c >> 5, col = c & 31;
                const int64_t gm = m0 + row, gk = k0 + col;
                const bool ok = gm < M && gk < kend;
                cp_async_4(a_s + (uint32_t)(row * AST + col) * 4u, ok ? A + gm * K + gk : A, ok ? 4 : 0);
            }
#pragma unroll 8
            for (int j = 0; j < BK * BN / THREADS; j++) {           // elements of B
                const int c = tid + j * THREADS;
                const int row = c >> 7, col = c & 127;
                const int64_t gk = k0 + row, gn = n0 + col;
                const bool ok = gk < kend && gn < N;
                cp_async_4(b_s + (uint32_t)(row * BN + col) * 4u, ok ? B + gk * N + gn : B, ok ? 4 : 0);
            }
        }
    };

    float acc[8][LT];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < LT; j++) acc[i][j] = 0.f;

#pragma unroll
    for (int st = 0; st < STAGES - 1; st++) {
        if (st < ntiles) load_stage(st, kbeg + (int64_t)st * BK);
        cp_async_commit();
    }
    for (int64_t t = 0; t < ntiles; t++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();                       // stage t landed; stage t - 1 is no longer read
        const int64_t tn = t + STAGES - 1;
        if (tn < ntiles) load_stage((int)(tn % STAGES), kbeg + tn * BK);
        cp_async_commit();
        const float* As = smem + (int)(t % STAGES) * STAGE_FLOATS;
        const float* Bs = As + A_FLOATS;
        const float* a_base = As + (wm * 64 + lm) * AST;
        const float* b_base = Bs + wn * WN + ln * 4;
        // Two of the eight four-k groups per loop body: a fully unrolled stage
        // outgrows the instruction cache.
#pragma unroll 2
        for (int k4 = 0; k4 < BK / 4; k4++) {
            float4 a[8];
#pragma unroll
            for (int i = 0; i < 8; i++) a[i] = *reinterpret_cast<const float4*>(a_base + i * 8 * AST + k4 * 4);
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                float b[LT];
#pragma unroll
                for (int j = 0; j < GN; j++) {
                    const float4 v = *reinterpret_cast<const float4*>(b_base + (k4 * 4 + kk) * BN + j * 16);
                    b[4 * j + 0] = v.x; b[4 * j + 1] = v.y; b[4 * j + 2] = v.z; b[4 * j + 3] = v.w;
                }
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const float av = kk == 0 ? a[i].x : kk == 1 ? a[i].y : kk == 2 ? a[i].z : a[i].w;
#pragma unroll
                    for (int j = 0; j < LT; j++) acc[i][j] = mac<FUSED>(av, b[j], acc[i][j]);
                }
            }
        }
    }
    cp_async_wait<0>();

    // Steps past kend multiplied zeros: the chains are those over [kbeg, kend).
    auto out_row = [&](int i) { return m0 + wm * 64 + lm + 8 * i; };
    auto out_col = [&](int g) { return n0 + wn * WN + ln * 4 + 16 * g; };
    simt_epilogue<8, GN>(p, acc, out_row, out_col, VEC, z, blockIdx.y * gridDim.x + blockIdx.x, last_flag);
}

// Grouped launch: one persistent kernel over a list of (problem, tile, K
// slice) units taken from an atomic counter, heaviest units first. Each unit
// is exactly the tile a per-GEMM launch of that problem computes, so results
// are identical to running the problems one by one.
template <int BM, int BN, bool FUSED>
__global__ void __launch_bounds__(kThreads, 2)
sgemm_simt_grouped_kernel(const GroupProblem* __restrict__ probs, const GroupUnit* __restrict__ units, int nunits,
                          unsigned* next) {
    __shared__ __align__(16) SimtSmem<BM, BN> sm;
    __shared__ int s_unit;
    for (;;) {
        if (threadIdx.x == 0) s_unit = (int)atomicAdd(next, 1u);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= nunits) break;
        const GroupUnit w = units[u];
        const GroupProblem& P = probs[w.problem];
        const unsigned tile = (unsigned)w.tm * (unsigned)P.tiles_n + (unsigned)w.tn;
        simt_tile<BM, BN, FUSED, 2>(P.a, (int64_t)w.tm * BM, (int64_t)w.tn * BN, w.z, tile, sm, P.vec != 0);
    }
}

// Split-K reduction for plans of three or more K slices: the slices wrote
// their partial products ([slice][M][N]); each thread sums one output over the
// slices in slice order -- the order of the in-kernel fixup and of the
// reference's panel sum C = p0 + p1 + ... -- so C is the same bit for bit. All
// outputs proceed in parallel, 16 slice loads in flight per thread, instead of
// one CTA per tile walking its slices in turn. HBM-bound: splits * M * N floats
// in, M * N out.
__global__ void __launch_bounds__(256)
simt_splitk_reduce_kernel(const float* __restrict__ partial, float* __restrict__ C, int64_t M, int64_t N,
                          int splits) {
    const size_t MN = (size_t)M * (size_t)N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)MN;
         i += (int64_t)gridDim.x * blockDim.x)
        C[i] = ordered_sum<64>(partial + i, MN, splits);
}

// Slices at or above which the partials are summed by the reduction kernel.
constexpr int kReduceAfterSplits = 3;

// Raises a kernel's dynamic shared memory limit once per device.
template <typename Kern>
cudaError_t smem_limit_once(Kern kern, int bytes, std::atomic<uint64_t>& done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && ((done.load() >> dev) & 1u)) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && dev < 64) done.fetch_or(1ull << dev);
    return e;
}

template <bool FUSED, bool VEC, int LT>
cudaError_t launch_cp_lt(const SimtArgs& a, dim3 grid, cudaStream_t s) {
    static std::atomic<uint64_t> done{0};
    cudaError_t e = smem_limit_once(sgemm_simt_cp_kernel<FUSED, VEC, LT>, cpk::SMEM, done);
    if (e != cudaSuccess) return e;
    sgemm_simt_cp_kernel<FUSED, VEC, LT><<<grid, cpk::Shape<LT>::THREADS, cpk::SMEM, s>>>(a);
    return cudaGetLastError();
}

// 8 x 16 outputs per thread: measured at 4096^3 (45.7 against 44.7 TFLOP/s)
// and 2048^3 (40.2 against 38.5) ahead of 8 x 8 with 256 threads.
template <bool FUSED, bool VEC>
cudaError_t launch_cp(const SimtArgs& a, dim3 grid, cudaStream_t s) {
    return launch_cp_lt<FUSED, VEC, 16>(a, grid, s);
}

template <int BM, int BN>
cudaError_t launch_tile(const SimtArgs& args, int variant, cudaStream_t s) {
    SimtArgs a = args;
    a.reduce_after = (a.splits >= kReduceAfterSplits) ? 1 : 0;
    dim3 grid((unsigned)((a.N + BN - 1) / BN), (unsigned)((a.M + BM - 1) / BM), (unsigned)a.splits);
    const bool vec = (a.K % 4 == 0) && (a.N % 4 == 0) &&
                     ((uintptr_t)a.A % 16 == 0) && ((uintptr_t)a.B % 16 == 0) && ((uintptr_t)a.C % 16 == 0);
    const bool fused = (variant != MAXMULSK_FP32_SCALAR);
    cudaError_t e;
    {
        PhaseScope ps(kPhaseGemm, s);
        if constexpr (BM == cpk::BM && BN == cpk::BN) {
            if (fused && vec) e = launch_cp<true, true>(a, grid, s);
            else if (fused) e = launch_cp<true, false>(a, grid, s);
            else if (vec) e = launch_cp<false, true>(a, grid, s);
            else e = launch_cp<false, false>(a, grid, s);
        } else {
            if (fused && vec) sgemm_simt_kernel<BM, BN, true, true><<<grid, kThreads, 0, s>>>(a);
            else if (fused) sgemm_simt_kernel<BM, BN, true, false><<<grid, kThreads, 0, s>>>(a);
            else if (vec) sgemm_simt_kernel<BM, BN, false, true><<<grid, kThreads, 0, s>>>(a);
            else sgemm_simt_kernel<BM, BN, false, false><<<grid, kThreads, 0, s>>>(a);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess || !a.reduce_after) return e;
    PhaseScope ps(kPhaseReduce, s);
    int64_t blocks = (a.M * a.N + 255) / 256;
    const int64_t cap = (int64_t)device_sm_count() * 8;
    if (cap > 0 && blocks > cap) blocks = cap;
    simt_splitk_reduce_kernel<<<(unsigned)blocks, 256, 0, s>>>(a.partial, a.C, a.M, a.N, a.splits);
    return cudaGetLastError();
}

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

size_t simt_workspace_bytes(int64_t M, int64_t K, int64_t N, int tile_m, int tile_n, int split_k) {
    const int splits = slice_count((size_t)K, split_k);
    if (splits <= 1) return 0;
    const size_t tiles = (size_t)((M + tile_m - 1) / tile_m) * (size_t)((N + tile_n - 1) / tile_n);
    return align256(tiles * sizeof(unsigned)) + align256((size_t)splits * (size_t)M * (size_t)N * sizeof(float));
}

bool simt_bind_workspace(SimtArgs& a, int tile_m, int tile_n, void* ws, size_t ws_bytes) {
    if (a.splits <= 1) { a.partial = nullptr; a.counters = nullptr; return true; }
    const size_t tiles = (size_t)((a.M + tile_m - 1) / tile_m) * (size_t)((a.N + tile_n - 1) / tile_n);
    const size_t need = align256(tiles * sizeof(unsigned)) + align256((size_t)a.splits * a.M * a.N * sizeof(float));
    if (!ws || ws_bytes < need) return false;
    a.counters = static_cast<unsigned*>(ws);
    a.partial = reinterpret_cast<float*>(static_cast<char*>(ws) + align256(tiles * sizeof(unsigned)));
    return true;
}

cudaError_t simt_launch(const SimtArgs& a, int tile_m, int tile_n, int variant, cudaStream_t s) {
    if (tile_m == 128 && tile_n == 128) return launch_tile<128, 128>(a, variant, s);
    if (tile_m == 128 && tile_n == 64) return launch_tile<128, 64>(a, variant, s);
    if (tile_m == 64 && tile_n == 64) return launch_tile<64, 64>(a, variant, s);
    return cudaErrorInvalidValue;
}

maxmulsk_status simt_run(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                         const maxmulsk_plan& plan, void* scratch, size_t scratch_bytes, cudaStream_t s) {
    SimtArgs a{};
    a.A = dA; a.B = dB; a.C = dC;
    a.M = (int64_t)M; a.K = (int64_t)K; a.N = (int64_t)N;
    a.kchunk = (int64_t)slice_len(K, plan.split_k);
    a.splits = slice_count(K, plan.split_k);
    if (!simt_bind_workspace(a, plan.tile_m, plan.tile_n, scratch, scratch_bytes)) {
        set_error_message("workspace too small for the SIMT plan");
        return MAXMULSK_ERR_INVALID;
    }
    if (a.splits > 1 && a.splits < kReduceAfterSplits) {
        // The split-K arrival counters must start at zero on every call (with
        // more slices, simt_splitk_reduce_kernel sums them and no counter is read).
        const size_t tiles = (size_t)((M + plan.tile_m - 1) / plan.tile_m) * ((N + plan.tile_n - 1) / plan.tile_n);
        maxmulsk_status st =
            cuda_status(cudaMemsetAsync(a.counters, 0, tiles * sizeof(unsigned), s), "cudaMemsetAsync(counters)");
        if (st != MAXMULSK_OK) return st;
    }
    return cuda_status(simt_launch(a, plan.tile_m, plan.tile_n, plan.variant, s), "sgemm_simt launch");
}

namespace {
template <int BM, int BN>
cudaError_t launch_grouped_tile(const GroupProblem* probs, const GroupUnit* units, int nunits, unsigned* next,
                                int grid, int variant, cudaStream_t s) {
    if (variant == MAXMULSK_FP32_SCALAR)
        sgemm_simt_grouped_kernel<BM, BN, false><<<grid, kThreads, 0, s>>>(probs, units, nunits, next);
    else
        sgemm_simt_grouped_kernel<BM, BN, true><<<grid, kThreads, 0, s>>>(probs, units, nunits, next);
    return cudaGetLastError();
}
}  // namespace

cudaError_t simt_grouped_launch(const GroupProblem* probs, const GroupUnit* units, int nunits, unsigned* next,
                                int tile_m, int tile_n, int variant, int grid, cudaStream_t s) {
    if (tile_m == 128 && tile_n == 128) return launch_grouped_tile<128, 128>(probs, units, nunits, next, grid, variant, s);
    if (tile_m == 128 && tile_n == 64) return launch_grouped_tile<128, 64>(probs, units, nunits, next, grid, variant, s);
    if (tile_m == 64 && tile_n == 64) return launch_grouped_tile<64, 64>(probs, units, nunits, next, grid, variant, s);
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Static-scratch variant: the split-K SIMT path with its counters and partial
// tiles in a fixed device array instead of caller or library allocations.
//
// Some callers cannot allocate device memory at the point of the call: a
// host application that owns the whole device memory budget and forbids its
// plug-ins to call cudaMalloc, or a latency-critical loop that cannot afford
// cudaMalloc/cudaFree (which may synchronise the device). For them this path
// allocates nothing: the scratch lives in the array below, which the module
// reserves on every GPU that loads this library and keeps until the process
// exits.
//
// Limits and rules:
//   * at most MAXMULSK_STATIC_SCRATCH_BYTES (16 MiB) of scratch: a plan that
//     needs more is rejected (MAXMULSK_ERR_UNSUPPORTED), C untouched;
//   * one array per device, shared by every call: calls that overlap on the
//     GPU (other streams, other host threads) race on it and must be
//     serialised by the caller;
//   * the first call on a device resolves the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture. The address is kept per CUDA context, so a
//     context made after cudaDeviceReset resolves it again (its first call,
//     too, belongs before any capture);
//   * the array keeps the last call's contents; the arrival counters that
//     must start at zero are cleared on the stream before every launch.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_simt_static_scratch[MAXMULSK_STATIC_SCRATCH_BYTES];

namespace {

// The array's device address is resolved once per CUDA context (the primary
// context of each device the library is used on), keyed on the context's
// process-unique id (cuCtxGetId), so a context created after cudaDeviceReset
// resolves it again instead of reusing an address that no longer exists.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct StaticAddr {
    int device;
    unsigned long long ctx_id;
    void* ptr;
};
std::mutex g_static_mu;
std::vector<StaticAddr> g_static_addr;

template <typename Fn>
Fn driver_fn(const char* name) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
        return reinterpret_cast<Fn>(p);
    return nullptr;
}

// Id of the current context (0 when the driver cannot say, which then keys
// the cache on the device alone).
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_ctx = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
    static CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_ctx && get_id && get_ctx(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
    return 0;
}

// Device address of g_simt_static_scratch in the current context. A thread
// with no context bound yet (id 0) resolves the address, which binds the
// device's primary context, and records it under that context's id.
cudaError_t static_scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (ctx != 0)
        for (const StaticAddr& a : g_static_addr)
            if (a.device == dev && a.ctx_id == ctx) { *out = a.ptr; return cudaSuccess; }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_simt_static_scratch);
    if (e != cudaSuccess) return e;
    ctx = current_context_id();
    for (StaticAddr& a : g_static_addr)
        if (a.device == dev) { a.ctx_id = ctx; a.ptr = p; *out = p; return cudaSuccess; }
    g_static_addr.push_back(StaticAddr{dev, ctx, p});
    *out = p;
    return cudaSuccess;
}

}  // namespace

maxmulsk_status simt_run_static_scratch(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                        const maxmulsk_plan& plan, cudaStream_t s) {
    maxmulsk_status st = classify_plan(M, K, N, &plan);
    if (st != MAXMULSK_OK) return st;
    if (plan.precision != MAXMULSK_PREC_FP32) {
        set_error_message("the static-scratch entry runs FP32 plans only");
        return MAXMULSK_ERR_UNSUPPORTED;
    }
    if (handle_empty_dev(dC, M, K, N, s, &st)) return st;
    if (!dA || !dB || !dC) { set_error_message("null matrix pointer"); return MAXMULSK_ERR_INVALID; }
    const size_t need = simt_workspace_bytes((int64_t)M, (int64_t)K, (int64_t)N, plan.tile_m, plan.tile_n, plan.split_k);
    if (need > (size_t)MAXMULSK_STATIC_SCRATCH_BYTES) {
        set_error_message("plan needs more scratch than the static maximum of MAXMULSK_STATIC_SCRATCH_BYTES (16 MiB)");
        return MAXMULSK_ERR_UNSUPPORTED;
    }
    void* base = nullptr;
    if (need > 0) {
        st = cuda_status(static_scratch_address(&base), "cudaGetSymbolAddress(static scratch)");
        if (st != MAXMULSK_OK) return st;
    }
    return simt_run(dA, dB, dC, M, K, N, plan, base, need, s);
}

}  // namespace mmsk
