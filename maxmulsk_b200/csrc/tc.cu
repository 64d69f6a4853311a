// Split-precision tensor-core GEMM for sm_100a (tcgen05 + TMEM + TMA).
//
// Replaces the reference's ZA outer-product micro-kernel and its driver
// (micro_kernel_1x4, sme/v3/sme-1x4-acc-kcout.cpp:215-346; run_multiplication_blocked
// :427-567) for the split-precision modes. C = A*B is formed as a sum of
// products of operand planes written by the split pre-pass (split.cu):
//   3xTF32 : hi*hi + hi*lo + lo*hi        (tcgen05.mma kind::tf32)
//   BF16x6 : l_i*l_j for i + j <= 2       (tcgen05.mma kind::f16, BF16)
//   BF16x9 : all nine l_i*l_j
// with every product accumulated in one FP32 accumulator in TMEM.
//
// Structure (one CTA per SM, persistent; 6 warps):
//   warp 0      TMA producer: per stage one 3-D load of all A planes
//               (128 x BK, K-major, 64-byte swizzle) and one 4-D load of all B
//               planes (BK x BN in 128-byte column panels, 128-byte swizzle),
//               into a ring of STAGES shared-memory stages.
//   warp 1      TMEM owner; one thread issues the MMAs (128 x BN x KSTEP) and
//               commits each stage back to the producer.
//   warps 2..5  epilogue: TMEM -> registers (tcgen05.ld 32x32b) -> global.
//               Two accumulators in TMEM let the epilogue of one tile overlap
//               the main loop of the next.
// Work units are (output tile, K slice) pairs; with several slices per tile,
// each slice writes a partial and the last slice to arrive (per 32-row
// quarter) sums the partials in slice order into C, deterministically
// (the reference's outer-Kc panel order, :464-471 and :530-558).
//
// Edges: the TMA boxes read zero outside the planes (M and K tails), the
// planes are zero-padded in K and N, and the epilogue predicates its stores,
// the counterpart of the reference's scratch-tile edge path (:539-558).
//
// Every wait on an mbarrier is bounded; on timeout the kernel records
// kErrTimeout in the device error word, stops issuing work, waits (bounded)
// for its own copies and MMAs in flight, frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>

#include "internal.hpp"
#include "sm100.cuh"

namespace mmsk {
namespace {

using namespace sm100;

template <int MODE, int BN>
struct Cfg {
    static constexpr bool TF32 = (MODE == MAXMULSK_PREC_3XTF32);
    static constexpr int P = TF32 ? 2 : 3;          // planes per operand
    static constexpr int ES = TF32 ? 4 : 2;         // bytes per plane element
    static constexpr int BM = 128;
    static constexpr int BK = 64 / ES;              // K per stage: A rows of 64 bytes
    static constexpr int KSTEP = 32 / ES;           // K per MMA (32 bytes)
    static constexpr int KSTEPS = BK / KSTEP;       // 2
    static constexpr int NBE = 128 / ES;            // N elements per 128-byte panel
    static constexpr int NBLK = BN / NBE;           // panels per tile
    static constexpr int A_PLANE = BM * 64;         // bytes of one A plane per stage
    static constexpr int B_PLANE = BK * BN * ES;    // bytes of one B plane per stage
    static constexpr int STAGE = P * (A_PLANE + B_PLANE);
    static constexpr int STAGES_RAW = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_RAW > 8 ? 8 : STAGES_RAW;
    static constexpr int SMEM = STAGES * STAGE + 1024;
    static constexpr int NPROD = TF32 ? 3 : (MODE == MAXMULSK_PREC_BF16X6 ? 6 : 9);
    static constexpr uint32_t IDESC = make_idesc(TF32 ? 2u : 1u, 128u, (uint32_t)BN);
    static constexpr uint32_t TMEM_COLS = 2 * BN;
    static_assert(STAGES >= 2, "not enough shared memory for two stages");
    static_assert(BN % NBE == 0, "tile_n must be a whole number of 128-byte panels");
};

// (A plane, B plane) of each product, in issue order.
__device__ __forceinline__ void product_planes(int mode, int q, int& pa, int& pb) {
    if (mode == MAXMULSK_PREC_3XTF32) {
        // hi*hi, hi*lo, lo*hi
        pa = (q == 2) ? 1 : 0;
        pb = (q == 1) ? 1 : 0;
    } else if (mode == MAXMULSK_PREC_BF16X6) {
        // (0,0) (0,1) (1,0) (0,2) (1,1) (2,0)
        const int ta[6] = {0, 0, 1, 0, 1, 2};
        const int tb[6] = {0, 1, 0, 2, 1, 0};
        pa = ta[q]; pb = tb[q];
    } else {
        pa = q / 3; pb = q % 3;
    }
}

struct TcParams {
    int64_t M, K, N;
    int64_t kchunk;
    int splits;
    int tiles_m, tiles_n;
    int64_t units;
    float* C;
    float* partial;
    unsigned* counters;      // 4 per tile (one per 32-row quarter)
    int* err;
    long long timeout;       // SM clocks per bounded wait
};

// Unit -> (tile row, tile column, slice). Slices of one tile are adjacent so
// they run at the same time; tiles are rastered in groups of 8 tile rows so
// concurrently running CTAs share A rows and B columns in L2.
__device__ __forceinline__ void decode_unit(const TcParams& p, int64_t u, int& tm, int& tn, int& z) {
    z = (int)(u % p.splits);
    const int64_t t = u / p.splits;
    constexpr int G = 8;
    const int64_t per_group = (int64_t)G * p.tiles_n;
    const int64_t g = t / per_group;
    const int64_t first_m = g * G;
    const int64_t gsz = min((int64_t)G, (int64_t)p.tiles_m - first_m);
    const int64_t r = t % per_group;
    tm = (int)(first_m + r % gsz);
    tn = (int)(r / gsz);
}

template <int MODE, int BN>
__global__ void __launch_bounds__(192, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const TcParams p) {
    using Cf = Cfg<MODE, BN>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[Cf::STAGES];
    __shared__ __align__(8) uint64_t empty_bar[Cf::STAGES];
    __shared__ __align__(8) uint64_t tfull_bar[2];
    __shared__ __align__(8) uint64_t tempty_bar[2];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < Cf::STAGES; s++) { mbar_init(&full_bar[s], 1); mbar_init(&empty_bar[s], 1); }
        for (int a = 0; a < 2; a++) { mbar_init(&tfull_bar[a], 1); mbar_init(&tempty_bar[a], 4); }
        mbar_init(&done_bar, 1);
        abort_s = 0;
        fence_mbar_init();
        fence_proxy_async();
    }
    if (warp == 0 && lane == 0) { prefetch_tmap(&tmA); prefetch_tmap(&tmB); }
    if (warp == 1) { tmem_alloc(&tmem_base_s, Cf::TMEM_COLS); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = tmem_base_s;

    auto fail = [&]() {
        atomicOr(p.err, kErrTimeout);
        abort_s = 1;
    };

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t issued = 0;
            for (int64_t u = blockIdx.x; u < p.units && !abort_s; u += gridDim.x) {
                int tm, tn, z;
                decode_unit(p, u, tm, tn, z);
                const int64_t kbeg = (int64_t)z * p.kchunk;
                const int64_t kend = min(p.K, kbeg + p.kchunk);
                const int64_t nkb = (kend - kbeg + Cf::BK - 1) / Cf::BK;
                bool ok = true;
                for (int64_t kb = 0; kb < nkb; kb++) {
                    if (!mbar_wait_bounded(&empty_bar[stage], phase ^ 1u, p.timeout)) { fail(); ok = false; break; }
                    if (abort_s) { ok = false; break; }
                    uint8_t* sa = smem + (size_t)stage * Cf::STAGE;
                    uint8_t* sb = sa + Cf::P * Cf::A_PLANE;
                    mbar_arrive_expect_tx(&full_bar[stage], (uint32_t)Cf::STAGE);
                    const int32_t k = (int32_t)(kbeg + kb * Cf::BK);
                    tma_load_3d(sa, &tmA, &full_bar[stage], k, tm * Cf::BM, 0);
                    tma_load_4d(sb, &tmB, &full_bar[stage], 0, k, tn * Cf::NBLK, 0);
                    issued++;
                    if (++stage == Cf::STAGES) { stage = 0; phase ^= 1u; }
                }
                if (!ok) break;
            }
            // No copy may still be landing in shared memory when the CTA exits.
            const int64_t first = issued > Cf::STAGES ? issued - Cf::STAGES : 0;
            for (int64_t j = first; j < issued; j++) {
                if (!mbar_wait_bounded(&full_bar[j % Cf::STAGES], (uint32_t)((j / Cf::STAGES) & 1), p.timeout)) {
                    atomicOr(p.err, kErrTimeout);
                    abort_s = 1;
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            for (int64_t u = blockIdx.x; u < p.units && !abort_s; u += gridDim.x) {
                int tm, tn, z;
                decode_unit(p, u, tm, tn, z);
                const int64_t kbeg = (int64_t)z * p.kchunk;
                const int64_t kend = min(p.K, kbeg + p.kchunk);
                const int64_t nkb = (kend - kbeg + Cf::BK - 1) / Cf::BK;
                if (!mbar_wait_bounded(&tempty_bar[acc], acc_phase ^ 1u, p.timeout)) { fail(); break; }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                bool ok = true;
                for (int64_t kb = 0; kb < nkb; kb++) {
                    if (!mbar_wait_bounded(&full_bar[stage], phase, p.timeout)) { fail(); ok = false; break; }
                    tc_fence_after();
                    const uint32_t a_base = smem_u32(smem + (size_t)stage * Cf::STAGE);
                    const uint32_t b_base = a_base + Cf::P * Cf::A_PLANE;
#pragma unroll
                    for (int ks = 0; ks < Cf::KSTEPS; ks++) {
#pragma unroll
                        for (int q = 0; q < Cf::NPROD; q++) {
                            int pa, pb;
                            product_planes(MODE, q, pa, pb);
                            const uint64_t adesc = make_smem_desc(
                                a_base + (uint32_t)(pa * Cf::A_PLANE + ks * 32), 16u, 512u, 4u);
                            const uint64_t bdesc = make_smem_desc(
                                b_base + (uint32_t)(pb * Cf::B_PLANE + ks * Cf::KSTEP * 128),
                                (uint32_t)(Cf::BK * 128), 1024u, 2u);
                            const uint32_t accum = (kb > 0 || ks > 0 || q > 0) ? 1u : 0u;
                            if constexpr (Cf::TF32) mma_tf32(d_tmem, adesc, bdesc, Cf::IDESC, accum);
                            else mma_bf16(d_tmem, adesc, bdesc, Cf::IDESC, accum);
                        }
                    }
                    tc_commit(&empty_bar[stage]);
                    if (++stage == Cf::STAGES) { stage = 0; phase ^= 1u; }
                }
                if (!ok) break;
                tc_commit(&tfull_bar[acc]);
                if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
            }
            // No MMA may still be running when TMEM is freed.
            tc_commit(&done_bar);
            if (!mbar_wait_bounded(&done_bar, 0u, p.timeout)) { atomicOr(p.err, kErrTimeout); abort_s = 1; }
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int quarter = warp & 3;                 // TMEM lanes 32*quarter .. +31
        const int64_t M = p.M, N = p.N;
        const size_t MN = (size_t)M * (size_t)N;
        const bool vec = (N % 4 == 0) && ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0) &&
                         (p.partial == nullptr || (reinterpret_cast<uintptr_t>(p.partial) & 15) == 0);
        int acc = 0;
        uint32_t acc_phase = 0;
        for (int64_t u = blockIdx.x; u < p.units; u += gridDim.x) {
            int stop = abort_s;
            int tm, tn, z;
            decode_unit(p, u, tm, tn, z);
            if (!stop && lane == 0) {
                if (!mbar_wait_bounded(&tfull_bar[acc], acc_phase, p.timeout)) { fail(); stop = 1; }
            }
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop) break;
            __syncwarp();
            tc_fence_after();
            const int64_t row = (int64_t)tm * Cf::BM + quarter * 32 + lane;
            const int64_t col0 = (int64_t)tn * BN;
            float* out = (p.splits > 1) ? p.partial + (size_t)z * MN : p.C;
#pragma unroll 1
            for (int c = 0; c < BN; c += 32) {
                uint32_t r[32];
                tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN + c), r);
                tmem_wait_ld();
                if (row < M) {
                    const int64_t cb = col0 + c;
                    float* dst = out + (size_t)row * (size_t)N + (size_t)cb;
                    if (vec && cb + 31 < N) {
#pragma unroll
                        for (int j = 0; j < 32; j += 4)
                            *reinterpret_cast<float4*>(dst + j) =
                                make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]),
                                            __uint_as_float(r[j + 2]), __uint_as_float(r[j + 3]));
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; j++)
                            if (cb + j < N) dst[j] = __uint_as_float(r[j]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty_bar[acc]);
            if (++acc == 2) { acc = 0; acc_phase ^= 1u; }

            if (p.splits > 1) {
                // This quarter's partial is written; the last slice to arrive
                // sums all slices in slice order.
                __threadfence();
                __syncwarp();
                int last = 0;
                const int64_t tile = (int64_t)tm * p.tiles_n + tn;
                unsigned* ctr = p.counters + tile * 4 + quarter;
                if (lane == 0) last = (atomicAdd(ctr, 1u) == (unsigned)(p.splits - 1));
                last = __shfl_sync(0xffffffffu, last, 0);
                if (last) {
                    __threadfence();
                    const int64_t r0 = (int64_t)tm * Cf::BM + quarter * 32;
                    for (int rr = 0; rr < 32; rr++) {
                        const int64_t rw = r0 + rr;
                        if (rw >= M) break;
                        for (int c = lane; c < BN; c += 32) {
                            const int64_t cc = col0 + c;
                            if (cc >= N) break;
                            const size_t off = (size_t)rw * (size_t)N + (size_t)cc;
                            float s = __ldcg(p.partial + off);
                            for (int q = 1; q < p.splits; q++) s = __fadd_rn(s, __ldcg(p.partial + (size_t)q * MN + off));
                            p.C[off] = s;
                        }
                    }
                    if (lane == 0) *ctr = 0u;
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, Cf::TMEM_COLS);
    }
}

// ---------------------------------------------------------------- host side
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
    });
    return fn;
}

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

size_t tiles_of(int64_t M, int64_t N, int tile_n) {
    return (size_t)((M + 127) / 128) * (size_t)((N + tile_n - 1) / tile_n);
}

template <int MODE, int BN>
cudaError_t launch_cfg(const TcArgs& a, cudaStream_t s) {
    using Cf = Cfg<MODE, BN>;
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const PlaneGeom g = plane_geom(a.M, a.K, a.N, a.precision);
    char* a_planes = static_cast<char*>(a.planes);
    char* b_planes = a_planes + (size_t)g.P * g.a_plane_bytes;
    const CUtensorMapDataType dt = Cf::TF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;

    CUtensorMap tmA, tmB;
    {
        const cuuint64_t dims[3] = {(cuuint64_t)g.Kp, (cuuint64_t)a.M, (cuuint64_t)g.P};
        const cuuint64_t strides[2] = {(cuuint64_t)g.Kp * Cf::ES, (cuuint64_t)g.a_plane_bytes};
        const cuuint32_t box[3] = {(cuuint32_t)Cf::BK, 128u, (cuuint32_t)Cf::P};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&tmA, dt, 3, a_planes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    {
        const cuuint64_t npan = (cuuint64_t)(g.Np / Cf::NBE);
        const cuuint64_t dims[4] = {(cuuint64_t)Cf::NBE, (cuuint64_t)a.K, npan, (cuuint64_t)g.P};
        const cuuint64_t strides[3] = {128u, (cuuint64_t)a.K * 128u, (cuuint64_t)g.b_plane_bytes};
        const cuuint32_t box[4] = {(cuuint32_t)Cf::NBE, (cuuint32_t)Cf::BK, (cuuint32_t)Cf::NBLK, (cuuint32_t)Cf::P};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        if (enc(&tmB, dt, 4, b_planes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }

    TcParams prm;
    prm.M = a.M; prm.K = a.K; prm.N = a.N;
    prm.kchunk = a.kchunk;
    prm.splits = a.splits;
    prm.tiles_m = (int)((a.M + 127) / 128);
    prm.tiles_n = (int)((a.N + BN - 1) / BN);
    prm.units = (int64_t)prm.tiles_m * prm.tiles_n * a.splits;
    prm.C = a.C;
    prm.partial = a.partial;
    prm.counters = a.counters;
    prm.err = a.err;
    prm.timeout = 2000000000LL;   // about one second at B200 clocks

    // Per device and cheap; set on every launch so every device gets it.
    cudaError_t e = cudaFuncSetAttribute(tc_gemm_kernel<MODE, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         Cf::SMEM);
    if (e != cudaSuccess) return e;
    const int sms = device_sm_count();
    const int64_t grid = prm.units < sms ? prm.units : sms;
    tc_gemm_kernel<MODE, BN><<<(unsigned)grid, 192, Cf::SMEM, s>>>(tmA, tmB, prm);
    return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_mode(const TcArgs& a, cudaStream_t s) {
    switch (a.tile_n) {
        case 64: return launch_cfg<MODE, 64>(a, s);
        case 128: return launch_cfg<MODE, 128>(a, s);
        case 256: return launch_cfg<MODE, 256>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

size_t tc_workspace_bytes(int64_t M, int64_t K, int64_t N, int precision, int tile_n, int split_k) {
    const PlaneGeom g = plane_geom(M, K, N, precision);
    size_t bytes = (size_t)g.P * (g.a_plane_bytes + g.b_plane_bytes);
    const int splits = slice_count((size_t)K, split_k);
    if (splits > 1) {
        bytes += align256(tiles_of(M, N, tile_n) * 4 * sizeof(unsigned));
        bytes += align256((size_t)splits * (size_t)M * (size_t)N * sizeof(float));
    }
    return align256(bytes);
}

bool tc_bind_workspace(TcArgs& a, void* ws, size_t ws_bytes) {
    const PlaneGeom g = plane_geom(a.M, a.K, a.N, a.precision);
    size_t need = (size_t)g.P * (g.a_plane_bytes + g.b_plane_bytes);
    if (a.splits > 1) {
        need += align256(tiles_of(a.M, a.N, a.tile_n) * 4 * sizeof(unsigned));
        need += align256((size_t)a.splits * (size_t)a.M * (size_t)a.N * sizeof(float));
    }
    if (!ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(ws) & 255) != 0) return false;
    char* base = static_cast<char*>(ws);
    a.planes = base;
    base += (size_t)g.P * (g.a_plane_bytes + g.b_plane_bytes);
    if (a.splits > 1) {
        a.counters = reinterpret_cast<unsigned*>(base);
        base += align256(tiles_of(a.M, a.N, a.tile_n) * 4 * sizeof(unsigned));
        a.partial = reinterpret_cast<float*>(base);
    } else {
        a.counters = nullptr;
        a.partial = nullptr;
    }
    return true;
}

cudaError_t tc_launch(const TcArgs& a, cudaStream_t s) {
    if (!a.reuse_planes) {
        cudaError_t e = split_launch(a.A, a.B, a.M, a.K, a.N, a.precision, a.planes, s);
        if (e != cudaSuccess) return e;
    }
    switch (a.precision) {
        case MAXMULSK_PREC_3XTF32: return launch_mode<MAXMULSK_PREC_3XTF32>(a, s);
        case MAXMULSK_PREC_BF16X6: return launch_mode<MAXMULSK_PREC_BF16X6>(a, s);
        case MAXMULSK_PREC_BF16X9: return launch_mode<MAXMULSK_PREC_BF16X9>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mmsk
