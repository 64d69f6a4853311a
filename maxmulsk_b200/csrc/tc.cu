// Split-precision tensor-core GEMM for sm_100a (tcgen05 + TMEM + TMA).
//
// Replaces the reference's ZA outer-product micro-kernel and its driver
// (micro_kernel_1x4, sme/v3/sme-1x4-acc-kcout.cpp:215-346; run_multiplication_blocked
// :427-567) for the split-precision modes. C = A*B is formed as a sum of
// products of operand planes written by the split pre-pass (split.cu):
//   3xTF32 : hi*hi + hi*lo + lo*hi        (tcgen05.mma kind::tf32)
//   BF16x6 : l_i*l_j for i + j <= 2       (tcgen05.mma kind::f16, BF16)
//   BF16x9 : all nine l_i*l_j
//
// Accuracy. The tensor cores accumulate in FP32 but lose low bits at every
// accumulation step, so the error of one long TMEM accumulation grows with its
// length (measured on B200: about 0.4 * L / sqrt(K) times the FP32 SIMT
// kernel's normwise error for a chain of L k's). The kernel therefore
// accumulates only a short chunk of k's in TMEM at a time (32, 128 or 256 by
// K: chunk_len, or the plan's chunk); the epilogue warps add each chunk into FP32 registers, round
// to nearest, chunk after chunk in k order. This is the reference's outer-Kc
// panel scheme (first panel stores, later panels add:
// sme/v3/sme-1x4-acc-kcout.cpp:464-471, :530-558) with a short panel, and it
// keeps the split modes at or near the SIMT kernel's error.
//
// Structure (one CTA per SM, persistent):
//   warp 0      TMA producer: per stage one 3-D load of all A planes
//               (128 x BK, K-major, 64-byte swizzle) and one load of all B
//               planes: K-major BN x BK with 64-byte swizzle (TF32), or
//               BK x BN in 128-byte column panels with 128-byte swizzle (BF16),
//               into a ring of STAGES shared-memory stages.
//   warp 1      TMEM owner; one thread issues the MMAs (128 x BN x KSTEP) of a
//               chunk into one of NACC TMEM accumulators (all 512 columns: 4
//               for tiles up to 128 columns wide, 2 for 256) and commits each
//               stage back to the producer and each chunk to the epilogue.
//   warps 2..   epilogue (4 or 8 warps): TMEM -> registers (tcgen05.ld
//               32x32b), chunk sums in registers, then the tile goes out
//               through swizzled shared-memory boxes and TMA stores (where the
//               boxes fit beside the ring: TMA_STORE) or straight from
//               registers. The MMAs run up to NACC - 1 chunks ahead of the
//               drain, so the drain's latency stays off the tensor pipe even
//               when a chunk is one stage long (K-split plans).
// Work units are (output tile, K slice) pairs; with several slices per tile,
// each slice writes a partial and the last slice to arrive (per warp's rows
// and columns) sums the partials in slice order into C, deterministically.
//
// Edges: the TMA boxes read zero outside the planes (M and K tails), the
// planes are zero-padded in K and N, and the epilogue's TMA store boxes are
// clipped at C's extent (register stores are predicated), the counterpart of
// the reference's scratch-tile edge path (:539-558).
//
// Every wait on an mbarrier is bounded; on timeout the kernel records
// kErrTimeout in the device error word, stops issuing work, waits (bounded)
// for its own copies and MMAs in flight, frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "internal.hpp"
#include "phase.hpp"
#include "sm100.cuh"
#include "split_math.cuh"

namespace mmsk {
int tc_slots(int precision, int tile_m, int tile_n);

namespace {

using namespace sm100;

// The TMA-store writeback stages one box of 32 rows x 32 FP32 columns
// (128-byte rows) per epilogue warp. Dynamic shared memory a CTA may use:
// 227 KB less 1 KB for the static barriers.
constexpr int kStoreBox = 32;
constexpr int kStoreWarpBytes = 32 * kStoreBox * 4;
constexpr int kSmemCap = 227 * 1024 - 1024;

template <int MODE, int BN>
struct Cfg {
    static constexpr bool TF32 = (MODE == MAXMULSK_PREC_3XTF32);
    static constexpr int P = TF32 ? 2 : 3;          // planes per operand
    static constexpr int ES = TF32 ? 4 : 2;         // bytes per plane element
    static constexpr int BM = 128;
    static constexpr int BK = 64 / ES;              // K per stage: A rows of 64 bytes
    static constexpr int KSTEP = 32 / ES;           // K per MMA (32 bytes)
    static constexpr int KSTEPS = BK / KSTEP;       // 2
    static constexpr bool B_KMAJOR = TF32;          // see make_idesc
    static constexpr int NBE = 128 / ES;            // N elements per 128-byte panel (N-major B)
    static constexpr int NBLK = BN / NBE;           // panels per tile (N-major B)
    static constexpr int A_PLANE = BM * 64;         // bytes of one A plane per stage
    static constexpr int B_PLANE = BK * BN * ES;    // bytes of one B plane per stage (BN rows of 64 B)
    static constexpr int STAGE = P * (A_PLANE + B_PLANE);
    static constexpr int STAGES_RAW = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_RAW > 8 ? 8 : STAGES_RAW;
    static constexpr int RING = STAGES * STAGE;
    static constexpr int NPROD = TF32 ? 3 : (MODE == MAXMULSK_PREC_BF16X6 ? 6 : 9);
    static constexpr uint32_t IDESC = make_idesc(TF32 ? 2u : 1u, 128u, (uint32_t)BN, B_KMAJOR ? 0u : 1u);
    static constexpr int NACC = (512 / BN) < 4 ? (512 / BN) : 4;   // TMEM accumulators
    static constexpr uint32_t TMEM_COLS = NACC * BN;
    // Epilogue: 4 warps per TMEM lane quarter set; 8 for tiles of 128 columns
    // or more (two column groups), so each thread drains 64 or 128 columns.
    static constexpr int EPI = (BN >= 128) ? 8 : 4;
    static constexpr int COLS = BN * 4 / EPI;        // columns per epilogue thread
    static constexpr int LDW = (COLS >= 128) ? 32 : 64;   // columns loaded per TMEM wait (register bound)
    static constexpr int THREADS = 64 + 32 * EPI;
    // TMA-store writeback where its staging fits beside the ring without
    // costing a stage (not BF16 tiles of 64 or 256 columns).
    static constexpr bool TMA_STORE = RING + 1024 + EPI * kStoreWarpBytes <= kSmemCap;
    static constexpr int SMEM = RING + 1024 + (TMA_STORE ? EPI * kStoreWarpBytes : 0);
    static_assert(STAGES >= 2, "not enough shared memory for two stages");
    static_assert(COLS % 32 == 0, "column split must be whole");
    static_assert(B_KMAJOR || NBLK * NBE == BN, "tile_n must be a whole number of 128-byte panels");
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
    int bm;                  // rows per tile: 128, or 256 for a CTA pair
    int tiles_m, tiles_n;
    // Schedule: tiles [0, main_tiles) are cut into main_splits K slices of
    // main_kchunk; tiles [main_tiles, tiles) into tail_splits slices of
    // tail_kchunk. Units are numbered main region first.
    int64_t tiles, main_tiles, main_units, units;
    int main_splits, tail_splits;
    int64_t main_kchunk, tail_kchunk;
    int max_splits;
    int chunk_kb;            // stages per TMEM accumulation chunk
    int reduce_after;        // split tiles only write partials; tc_splitk_reduce_kernel sums them
    int store_c;             // whole tiles leave through the C tensor map (TMA stores)
    float* C;
    float* partial;          // [split tile][slice][BN columns x 128 rows], column-major, split tiles only
    unsigned* counters;      // EPI per split tile (one per epilogue warp)
    int* err;
    long long timeout;       // SM clocks per bounded wait
};

struct Unit {
    int tm, tn, z, nsplit;
    int64_t kbeg, kend;
    int64_t sti;             // index among split tiles, -1 when the tile is whole
};

// Tile t -> (tile row, tile column), rastered in groups of 8 tile rows so
// concurrently running CTAs share A rows and B columns in L2. I is the index
// type: 32-bit unsigned division is a few instructions, 64-bit division a
// long software routine at the start of every unit.
template <typename I>
__device__ __forceinline__ void tile_coords_t(const TcParams& p, I t, int& tm, int& tn) {
    constexpr I G = 8;
    const I per_group = G * (I)p.tiles_n;
    const I g = t / per_group;
    const I first_m = g * G;
    const I gsz = min(G, (I)p.tiles_m - first_m);
    const I r = t % per_group;
    tm = (int)(first_m + r % gsz);
    tn = (int)(r / gsz);
}

template <typename I>
__device__ __forceinline__ Unit decode_unit_t(const TcParams& p, I u) {
    Unit w;
    I t;
    int64_t kc;
    if (u < (I)p.main_units) {
        w.z = (int)(u % (I)p.main_splits);
        t = u / (I)p.main_splits;
        w.nsplit = p.main_splits;
        kc = p.main_kchunk;
        w.sti = (p.main_splits > 1) ? (int64_t)t : -1;
    } else {
        const I v = u - (I)p.main_units;
        w.z = (int)(v % (I)p.tail_splits);
        t = (I)p.main_tiles + v / (I)p.tail_splits;
        w.nsplit = p.tail_splits;
        kc = p.tail_kchunk;
        w.sti = (p.tail_splits > 1) ? (int64_t)(t - (I)p.main_tiles) : -1;
    }
    w.kbeg = (int64_t)w.z * kc;
    w.kend = min(p.K, w.kbeg + kc);
    tile_coords_t<I>(p, t, w.tm, w.tn);
    return w;
}

// Unit -> its tile, K slice and where its partial goes. Slices of one tile
// are adjacent so they run at the same time.
__device__ __forceinline__ Unit decode_unit(const TcParams& p, int64_t u) {
    if (p.units <= (int64_t)UINT32_MAX) return decode_unit_t<uint32_t>(p, (uint32_t)u);
    return decode_unit_t<uint64_t>(p, (uint64_t)u);
}

// What the roles of a persistent kernel need to know about one work unit:
// its tile and K slice, and the problem it belongs to.
struct UnitView {
    Unit w;
    int problem;             // index in a grouped launch (0 for one GEMM)
    int64_t M, N;
    float* C;
    float* partial;          // the problem's partial tiles: [split tile][slice][BN x 128], column-major
    unsigned* counters;      // the problem's arrival counters: EPI per split tile
    int max_splits;          // slices per split tile in the partial layout
    int chunk_kb;            // stages per TMEM accumulation chunk
    int reduce_after;        // partials are summed by tc_splitk_reduce_kernel
};

// Units of one GEMM (the schedule in TcParams).
struct SingleSrc {
    const TcParams& p;
    const CUtensorMap* tmC = nullptr;    // C for the TMA-store writeback, or none
    __device__ __forceinline__ int64_t units() const { return p.units; }
    __device__ __forceinline__ const CUtensorMap* store_map(const UnitView&) const { return tmC; }
    // The r-th unit of this CTA: units are dealt round-robin.
    __device__ __forceinline__ int64_t unit_of(int64_t r) const { return r * gridDim.x + blockIdx.x; }
    __device__ __forceinline__ void get(int64_t u, UnitView& v) const {
        v.w = decode_unit(p, u);
        v.problem = 0;
        v.M = p.M; v.N = p.N; v.C = p.C; v.partial = p.partial; v.counters = p.counters;
        v.max_splits = p.max_splits; v.chunk_kb = p.chunk_kb; v.reduce_after = p.reduce_after;
    }
    __device__ __forceinline__ const void* map_a(const UnitView&, const void* single) const { return single; }
    __device__ __forceinline__ const void* map_b(const UnitView&, const void* single) const { return single; }
    __device__ __forceinline__ void acquire(const void*, const void*) const {}
};

// One epilogue warp's 32 rows x COLS sums (thread `lane` holds row row0 +
// lane, columns col0 ..) -> C by TMEM -> registers -> shared memory -> TMA
// store, in boxes of 32 columns: the warp writes a box into `buf` with the
// 128-byte swizzle (16-byte chunk c of row r at chunk c ^ (r & 7), so the
// eight rows of each quarter-warp store hit eight different bank groups),
// makes it visible to the async proxy, and lane 0 stores it. The box is
// clipped at C's extent, so rows >= M and columns >= N are never written.
// Before `buf` is rewritten lane 0 waits until its previous store has read
// it; the caller waits for all of them before the CTA exits.
template <int COLS>
__device__ __forceinline__ void store_rows_tma(const CUtensorMap* tmC, uint8_t* buf, const float (&sum)[COLS],
                                               int lane, int64_t row0, int64_t col0, int64_t M, int64_t N) {
    if (row0 >= M) return;
#pragma unroll
    for (int b = 0; b < COLS; b += kStoreBox) {
        if (col0 + b < N) {
            if (lane == 0) bulk_wait_read_all();
            __syncwarp();
            uint8_t* rowp = buf + lane * (kStoreBox * 4);
#pragma unroll
            for (int c = 0; c < kStoreBox / 4; c++)
                *reinterpret_cast<float4*>(rowp + ((c ^ (lane & 7)) << 4)) =
                    make_float4(sum[b + 4 * c], sum[b + 4 * c + 1], sum[b + 4 * c + 2], sum[b + 4 * c + 3]);
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) {
                tma_store_2d(tmC, buf, (int32_t)(col0 + b), (int32_t)row0);
                bulk_commit_group();
            }
        }
    }
}

// One thread's row segment of C (COLS columns from col0) from registers:
// 128-bit stores where the segment and C allow them, else element by element
// up to N. A row past M writes nothing.
template <int COLS>
__device__ __forceinline__ void store_row_regs(const float (&sum)[COLS], float* C, int64_t row, int64_t col0,
                                               int64_t M, int64_t N, bool vec) {
    if (row >= M) return;
    float* dst = C + (size_t)row * (size_t)N + (size_t)col0;
    if (vec && col0 + COLS <= N) {
#pragma unroll
        for (int j = 0; j < COLS; j += 4)
            *reinterpret_cast<float4*>(dst + j) = make_float4(sum[j], sum[j + 1], sum[j + 2], sum[j + 3]);
    } else {
#pragma unroll
        for (int j = 0; j < COLS; j++)
            if (col0 + j < N) dst[j] = sum[j];
    }
}

// A K slice z of a split tile: this thread's row segment goes into the
// slice's partial tile (`seg` = the segment's first element in slice 0;
// slices `tile` floats apart). Partial tiles are column-major, 128 rows per
// column (element (r, c) at c * 128 + r), so the 32 lanes of a warp, 32
// consecutive rows, store each column as one contiguous 128-byte line.
// Unless a reduction kernel sums the slices (`reduce_after`), the last slice
// to arrive on this warp's counter reads every slice back in slice order (its
// own included), sums them with round-to-nearest adds, stores the segment of
// C and resets the counter.
template <int COLS>
__device__ __forceinline__ void finish_slice(float (&sum)[COLS], float* seg, size_t tile, int z, int nsplit,
                                             bool reduce_after, unsigned* ctr, int lane, float* C, int64_t row,
                                             int64_t col0, int64_t M, int64_t N, bool vec) {
    float* part = seg + (size_t)z * tile;
#pragma unroll
    for (int j = 0; j < COLS; j++) __stcg(part + (size_t)j * 128, sum[j]);
    if (reduce_after) return;
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane == 0) last = (atomicAdd(ctr, 1u) == (unsigned)(nsplit - 1));
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
#pragma unroll
    for (int j = 0; j < COLS; j++) sum[j] = __ldcg(seg + (size_t)j * 128);
    for (int q = 1; q < nsplit; q++) {
        const float* bq = seg + (size_t)q * tile;
#pragma unroll
        for (int j = 0; j < COLS; j++) sum[j] = __fadd_rn(sum[j], __ldcg(bq + (size_t)j * 128));
    }
    store_row_regs<COLS>(sum, C, row, col0, M, N, vec);
    if (lane == 0) *ctr = 0u;
}

// Epilogue warps of the one-CTA kernels: each TMEM chunk of a unit is drained
// into FP32 register sums (round to nearest, chunk after chunk in k order);
// then the unit's tile is stored (by TMA stores through this warp's
// buffer `cbuf` when the source gives a C tensor map, else from registers), or, for
// a K slice, its partial tile, and the last slice to arrive sums all slices
// in slice order (unless a separate reduction kernel does that).
template <class Cf, int BN, class Src>
__device__ __forceinline__ void epilogue_role(const Src& src, int* err, long long timeout, uint32_t tmem_base,
                                              uint64_t* tfull_bar, uint64_t* tempty_bar, volatile int& abort_s,
                                              int warp, int lane, uint8_t* cbuf) {
    constexpr int COLS = Cf::COLS;                   // columns of one epilogue thread
    auto fail = [&]() {
        atomicOr(err, kErrTimeout);
        abort_s = 1;
    };
    auto kblocks = [&](const Unit& w) -> int64_t { return (w.kend - w.kbeg + Cf::BK - 1) / Cf::BK; };
    const int ew = warp - 2;                      // epilogue warp 0 .. EPI-1
    const int quarter = warp & 3;                 // TMEM lanes 32*quarter .. +31
    const int cgroup = ew / 4;                    // which COLS-wide column group
    int acc = 0;
    uint32_t acc_phase = 0;
    float sum[COLS];
    bool stop = false;
    for (int64_t round = 0, u = src.unit_of(0); u < src.units() && !stop; u = src.unit_of(++round)) {
        UnitView v;
        src.get(u, v);
        const Unit& w = v.w;
        const int64_t M = v.M, N = v.N;
        const bool vec = (N % 4 == 0) && ((reinterpret_cast<uintptr_t>(v.C) & 15) == 0) &&
                         (v.partial == nullptr || (reinterpret_cast<uintptr_t>(v.partial) & 15) == 0);
        const int64_t nkb = kblocks(w);
        for (int64_t kb0 = 0; kb0 < nkb; kb0 += v.chunk_kb) {
            int bad = abort_s;
            if (!bad && lane == 0) {
                if (!mbar_wait_bounded(&tfull_bar[acc], acc_phase, timeout)) { fail(); bad = 1; }
            }
            bad = __shfl_sync(0xffffffffu, bad, 0);
            if (bad) { stop = true; break; }
            tc_fence_after();
            const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN + cgroup * COLS);
#pragma unroll
            for (int c = 0; c < COLS; c += Cf::LDW) {
                uint32_t r[Cf::LDW];
                if constexpr (Cf::LDW == 16) {
                    tmem_ld_32x32b_x16(taddr + (uint32_t)c, r);
                } else {
#pragma unroll
                    for (int h = 0; h < Cf::LDW; h += 32)
                        tmem_ld_32x32b_x32(taddr + (uint32_t)(c + h), *reinterpret_cast<uint32_t(*)[32]>(&r[h]));
                }
                tmem_wait_ld();
                if (kb0 == 0) {
#pragma unroll
                    for (int j = 0; j < Cf::LDW; j++) sum[c + j] = __uint_as_float(r[j]);
                } else {
#pragma unroll
                    for (int j = 0; j < Cf::LDW; j++) sum[c + j] = __fadd_rn(sum[c + j], __uint_as_float(r[j]));
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty_bar[acc]);
            if (++acc == Cf::NACC) { acc = 0; acc_phase ^= 1u; }
        }
        if (stop) break;

        // ---- the unit's sums are complete: store them
        const int lrow = quarter * 32 + lane;             // row within the tile
        const int lcol = cgroup * COLS;                   // first column within the tile
        const int64_t row = (int64_t)w.tm * Cf::BM + lrow;
        const int64_t col0 = (int64_t)w.tn * BN + lcol;
        if (w.sti < 0) {
            const CUtensorMap* tmC = src.store_map(v);
            if (cbuf && tmC) store_rows_tma<COLS>(tmC, cbuf, sum, lane, row - lane, col0, M, N);
            else store_row_regs<COLS>(sum, v.C, row, col0, M, N, vec);
            continue;
        }
        constexpr size_t TILE = (size_t)Cf::BM * BN;
        finish_slice<COLS>(sum, v.partial + (size_t)w.sti * v.max_splits * TILE + (size_t)lcol * 128 + lrow, TILE, w.z,
                           w.nsplit, v.reduce_after != 0, v.counters + (size_t)w.sti * Cf::EPI + ew, lane, v.C, row,
                           col0, M, N, vec);
    }
    // This warp's TMA stores have completed before the CTA exits.
    if (cbuf && lane == 0) bulk_wait_all();
}

template <int MODE, int BN>
__global__ void __launch_bounds__(Cfg<MODE, BN>::THREADS, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const __grid_constant__ CUtensorMap tmC, const TcParams p) {
    using Cf = Cfg<MODE, BN>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[Cf::STAGES];
    __shared__ __align__(8) uint64_t empty_bar[Cf::STAGES];
    __shared__ __align__(8) uint64_t tfull_bar[Cf::NACC];
    __shared__ __align__(8) uint64_t tempty_bar[Cf::NACC];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < Cf::STAGES; s++) { mbar_init(&full_bar[s], 1); mbar_init(&empty_bar[s], 1); }
        for (int a = 0; a < Cf::NACC; a++) { mbar_init(&tfull_bar[a], 1); mbar_init(&tempty_bar[a], Cf::EPI); }
        mbar_init(&done_bar, 1);
        abort_s = 0;
        fence_mbar_init();
        fence_proxy_async();
    }
    if (warp == 0 && lane == 0) {
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
        if (p.store_c) prefetch_tmap(&tmC);
    }
    if (warp == 1) { tmem_alloc(&tmem_base_s, Cf::TMEM_COLS); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = tmem_base_s;

    auto fail = [&]() {
        atomicOr(p.err, kErrTimeout);
        abort_s = 1;
    };
    auto kblocks = [&](const Unit& w) -> int64_t { return (w.kend - w.kbeg + Cf::BK - 1) / Cf::BK; };

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t issued = 0;
            for (int64_t u = blockIdx.x; u < p.units && !abort_s; u += gridDim.x) {
                const Unit w = decode_unit(p, u);
                const int64_t nkb = kblocks(w);
                bool ok = true;
                for (int64_t kb = 0; kb < nkb; kb++) {
                    if (!mbar_wait_bounded(&empty_bar[stage], phase ^ 1u, p.timeout)) { fail(); ok = false; break; }
                    if (abort_s) { ok = false; break; }
                    uint8_t* sa = smem + (size_t)stage * Cf::STAGE;
                    uint8_t* sb = sa + Cf::P * Cf::A_PLANE;
                    mbar_arrive_expect_tx(&full_bar[stage], (uint32_t)Cf::STAGE);
                    const int32_t k = (int32_t)(w.kbeg + kb * Cf::BK);
                    tma_load_3d(sa, &tmA, &full_bar[stage], k, w.tm * Cf::BM, 0);
                    if constexpr (Cf::B_KMAJOR) tma_load_3d(sb, &tmB, &full_bar[stage], k, w.tn * BN, 0);
                    else tma_load_4d(sb, &tmB, &full_bar[stage], 0, k, w.tn * Cf::NBLK, 0);
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
            bool ok = true;
            for (int64_t u = blockIdx.x; u < p.units && ok && !abort_s; u += gridDim.x) {
                const int64_t nkb = kblocks(decode_unit(p, u));
                for (int64_t kb0 = 0; kb0 < nkb && ok; kb0 += p.chunk_kb) {
                    // one chunk of up to CHUNK_KB stages into accumulator `acc`
                    if (!mbar_wait_bounded(&tempty_bar[acc], acc_phase ^ 1u, p.timeout)) { fail(); ok = false; break; }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                    const int64_t kb1 = min(nkb, kb0 + (int64_t)p.chunk_kb);
                    for (int64_t kb = kb0; kb < kb1; kb++) {
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
                                const uint64_t bdesc = Cf::B_KMAJOR
                                    ? make_smem_desc(b_base + (uint32_t)(pb * Cf::B_PLANE + ks * 32), 16u, 512u, 4u)
                                    : make_smem_desc(b_base + (uint32_t)(pb * Cf::B_PLANE + ks * Cf::KSTEP * 128),
                                                     (uint32_t)(Cf::BK * 128), 1024u, 2u);
                                const uint32_t accum = (kb > kb0 || ks > 0 || q > 0) ? 1u : 0u;
                                if constexpr (Cf::TF32) mma_tf32(d_tmem, adesc, bdesc, Cf::IDESC, accum);
                                else mma_bf16(d_tmem, adesc, bdesc, Cf::IDESC, accum);
                            }
                        }
                        tc_commit(&empty_bar[stage]);
                        if (++stage == Cf::STAGES) { stage = 0; phase ^= 1u; }
                    }
                    if (!ok) break;
                    tc_commit(&tfull_bar[acc]);
                    if (++acc == Cf::NACC) { acc = 0; acc_phase ^= 1u; }
                }
            }
            // No MMA may still be running when TMEM is freed.
            tc_commit(&done_bar);
            if (!mbar_wait_bounded(&done_bar, 0u, p.timeout)) { atomicOr(p.err, kErrTimeout); abort_s = 1; }
        }
    } else {
        // ------------------------------------------------------------ epilogue
        uint8_t* cbuf = (Cf::TMA_STORE && p.store_c) ? smem + Cf::RING + (warp - 2) * kStoreWarpBytes : nullptr;
        epilogue_role<Cf, BN>(SingleSrc{p, p.store_c ? &tmC : nullptr}, p.err, p.timeout, tmem_base, tfull_bar,
                              tempty_bar, abort_s, warp, lane, cbuf);
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, Cf::TMEM_COLS);
    }
}

// ============================================================================
// CTA-pair variant (tcgen05 cta_group::2). Two CTAs of a cluster share one
// 256 x BN tile: each stages its own 128 rows of A and its own BN/2 columns of
// B, the leader CTA (rank 0) issues 256 x BN x KSTEP MMAs that read both CTAs'
// shared memory and write each CTA's 128 rows into that CTA's TMEM. Per SM
// this halves the B operand traffic from L2 and shared memory. The epilogue is
// the single-CTA one, per CTA. Loads are plain (no multicast); only the MMA
// commit arrives on both CTAs' barriers.
// ============================================================================
template <int MODE, int BN>
struct CfgPair {
    static constexpr bool TF32 = (MODE == MAXMULSK_PREC_3XTF32);
    static constexpr int P = TF32 ? 2 : 3;
    static constexpr int ES = TF32 ? 4 : 2;
    static constexpr int BM = 256;                   // rows per pair tile
    static constexpr int HM = 128;                   // rows per CTA
    static constexpr int HN = BN / 2;                // B columns per CTA
    static constexpr int BK = 64 / ES;
    static constexpr int KSTEP = 32 / ES;
    static constexpr int KSTEPS = BK / KSTEP;
    static constexpr bool B_KMAJOR = TF32;
    static constexpr int NBE = 128 / ES;
    static constexpr int HNBLK = HN / NBE;           // B panels per CTA (N-major B)
    static constexpr int A_PLANE = HM * 64;
    static constexpr int B_PLANE = BK * HN * ES;
    static constexpr int STAGE = P * (A_PLANE + B_PLANE);
    static constexpr int STAGES_RAW = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_RAW > 8 ? 8 : STAGES_RAW;
    static constexpr int RING = STAGES * STAGE;
    static constexpr int NPROD = TF32 ? 3 : (MODE == MAXMULSK_PREC_BF16X6 ? 6 : 9);
    static constexpr uint32_t IDESC = make_idesc(TF32 ? 2u : 1u, 256u, (uint32_t)BN, B_KMAJOR ? 0u : 1u);
    static constexpr uint32_t TMEM_COLS = 2 * BN;
    static constexpr int EPI = (BN >= 128) ? 8 : 4;
    static constexpr int COLS = BN * 4 / EPI;
    static constexpr int LDW = (COLS >= 128) ? 32 : 64;
    static constexpr int THREADS = 64 + 32 * EPI;
    static constexpr bool TMA_STORE = RING + 1024 + EPI * kStoreWarpBytes <= kSmemCap;   // as Cfg
    static constexpr int SMEM = RING + 1024 + (TMA_STORE ? EPI * kStoreWarpBytes : 0);
    static_assert(STAGES >= 2, "not enough shared memory for two stages");
    static_assert(B_KMAJOR || HNBLK * NBE == HN, "half tile must be whole 128-byte panels");
    static_assert(COLS % 32 == 0, "column split must be whole");
};

template <int MODE, int BN>
__global__ void __launch_bounds__(CfgPair<MODE, BN>::THREADS, 1)
tc_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ CUtensorMap tmC, const TcParams p) {
    using Cf = CfgPair<MODE, BN>;
    constexpr int COLS = Cf::COLS;
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
    const uint32_t rank = cluster_ctarank() & 1u;
    const bool leader = (rank == 0);
    const int64_t pair = blockIdx.x >> 1;
    const int64_t npairs = gridDim.x >> 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < Cf::STAGES; s++) { mbar_init(&full_bar[s], 1); mbar_init(&empty_bar[s], 1); }
        for (int a = 0; a < 2; a++) { mbar_init(&tfull_bar[a], 1); mbar_init(&tempty_bar[a], 2 * Cf::EPI); }
        mbar_init(&done_bar, 1);
        abort_s = 0;
        fence_mbar_init();
        fence_proxy_async();
    }
    if (warp == 0 && lane == 0) {
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
        if (p.store_c) prefetch_tmap(&tmC);
    }
    if (warp == 1) { tmem_alloc_pair(&tmem_base_s, Cf::TMEM_COLS); tmem_relinquish_pair(); }
    tc_fence_before();
    cluster_sync();                 // barriers of both CTAs initialised before any remote use
    tc_fence_after();
    const uint32_t tmem_base = tmem_base_s;

    auto fail = [&]() {
        atomicOr(p.err, kErrTimeout);
        abort_s = 1;
    };
    auto kblocks = [&](const Unit& w) -> int64_t { return (w.kend - w.kbeg + Cf::BK - 1) / Cf::BK; };

    if (warp == 0) {
        // ------------------------------------------------------------ producer (both CTAs)
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t issued = 0;
            for (int64_t u = pair; u < p.units && !abort_s; u += npairs) {
                const Unit w = decode_unit(p, u);
                const int64_t nkb = kblocks(w);
                bool ok = true;
                for (int64_t kb = 0; kb < nkb; kb++) {
                    if (!mbar_wait_bounded(&empty_bar[stage], phase ^ 1u, p.timeout)) { fail(); ok = false; break; }
                    if (abort_s) { ok = false; break; }
                    uint8_t* sa = smem + (size_t)stage * Cf::STAGE;
                    uint8_t* sb = sa + Cf::P * Cf::A_PLANE;
                    const uint32_t bar = mapa_shared(&full_bar[stage], 0);   // the leader's barrier
                    if (leader) mbar_arrive_expect_tx(&full_bar[stage], (uint32_t)(2 * Cf::STAGE));
                    const int32_t k = (int32_t)(w.kbeg + kb * Cf::BK);
                    tma_load_3d_pair(sa, &tmA, bar, k, w.tm * Cf::BM + (int32_t)rank * Cf::HM, 0);
                    if constexpr (Cf::B_KMAJOR)
                        tma_load_3d_pair(sb, &tmB, bar, k, w.tn * BN + (int32_t)rank * Cf::HN, 0);
                    else
                        tma_load_4d_pair(sb, &tmB, bar, 0, k, w.tn * (BN / Cf::NBE) + (int32_t)rank * Cf::HNBLK, 0);
                    issued++;
                    if (++stage == Cf::STAGES) { stage = 0; phase ^= 1u; }
                }
                if (!ok) break;
            }
            // The leader's full barriers count both CTAs' copies: wait for ours
            // there (leader) or for the MMAs to release our stages (follower),
            // so no copy into this CTA's shared memory is still in flight.
            const int64_t first = issued > Cf::STAGES ? issued - Cf::STAGES : 0;
            for (int64_t j = first; j < issued; j++) {
                const int st = (int)(j % Cf::STAGES);
                const uint32_t par = (uint32_t)((j / Cf::STAGES) & 1);
                const bool okw = leader ? mbar_wait_bounded(&full_bar[st], par, p.timeout)
                                        : mbar_wait_bounded(&empty_bar[st], par, p.timeout);
                if (!okw) { atomicOr(p.err, kErrTimeout); abort_s = 1; }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer (leader only)
        if (lane == 0 && leader) {
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            bool ok = true;
            for (int64_t u = pair; u < p.units && ok && !abort_s; u += npairs) {
                const int64_t nkb = kblocks(decode_unit(p, u));
                for (int64_t kb0 = 0; kb0 < nkb && ok; kb0 += p.chunk_kb) {
                    if (!mbar_wait_bounded(&tempty_bar[acc], acc_phase ^ 1u, p.timeout)) { fail(); ok = false; break; }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                    const int64_t kb1 = min(nkb, kb0 + (int64_t)p.chunk_kb);
                    for (int64_t kb = kb0; kb < kb1; kb++) {
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
                                const uint64_t bdesc = Cf::B_KMAJOR
                                    ? make_smem_desc(b_base + (uint32_t)(pb * Cf::B_PLANE + ks * 32), 16u, 512u, 4u)
                                    : make_smem_desc(b_base + (uint32_t)(pb * Cf::B_PLANE + ks * Cf::KSTEP * 128),
                                                     (uint32_t)(Cf::BK * 128), 1024u, 2u);
                                const uint32_t accum = (kb > kb0 || ks > 0 || q > 0) ? 1u : 0u;
                                if constexpr (Cf::TF32) mma_tf32_pair(d_tmem, adesc, bdesc, Cf::IDESC, accum);
                                else mma_bf16_pair(d_tmem, adesc, bdesc, Cf::IDESC, accum);
                            }
                        }
                        tc_commit_pair_multicast(&empty_bar[stage], (uint16_t)0x3);
                        if (++stage == Cf::STAGES) { stage = 0; phase ^= 1u; }
                    }
                    if (!ok) break;
                    tc_commit_pair_multicast(&tfull_bar[acc], (uint16_t)0x3);
                    if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
                }
            }
            tc_commit_pair(&done_bar);
            if (!mbar_wait_bounded(&done_bar, 0u, p.timeout)) { atomicOr(p.err, kErrTimeout); abort_s = 1; }
        }
    } else {
        // ------------------------------------------------------------ epilogue (both CTAs)
        const int ew = warp - 2;
        const int quarter = warp & 3;
        const int cgroup = ew / 4;
        uint8_t* cbuf = (Cf::TMA_STORE && p.store_c) ? smem + Cf::RING + ew * kStoreWarpBytes : nullptr;
        const int64_t M = p.M, N = p.N;
        const bool vec = (N % 4 == 0) && ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0);
        const uint32_t tempty_leader0 = mapa_shared(&tempty_bar[0], 0);
        const uint32_t tempty_leader1 = mapa_shared(&tempty_bar[1], 0);
        int acc = 0;
        uint32_t acc_phase = 0;
        float sum[COLS];
        bool stop = false;
        for (int64_t u = pair; u < p.units && !stop; u += npairs) {
            const Unit w = decode_unit(p, u);
            const int64_t nkb = kblocks(w);
            for (int64_t kb0 = 0; kb0 < nkb; kb0 += p.chunk_kb) {
                int bad = abort_s;
                if (!bad && lane == 0) {
                    if (!mbar_wait_bounded(&tfull_bar[acc], acc_phase, p.timeout)) { fail(); bad = 1; }
                }
                bad = __shfl_sync(0xffffffffu, bad, 0);
                if (bad) { stop = true; break; }
                tc_fence_after();
                const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN + cgroup * COLS);
#pragma unroll
                for (int c = 0; c < COLS; c += Cf::LDW) {
                    uint32_t r[Cf::LDW];
#pragma unroll
                    for (int h = 0; h < Cf::LDW; h += 32)
                        tmem_ld_32x32b_x32(taddr + (uint32_t)(c + h), *reinterpret_cast<uint32_t(*)[32]>(&r[h]));
                    tmem_wait_ld();
                    if (kb0 == 0) {
#pragma unroll
                        for (int j = 0; j < Cf::LDW; j++) sum[c + j] = __uint_as_float(r[j]);
                    } else {
#pragma unroll
                        for (int j = 0; j < Cf::LDW; j++) sum[c + j] = __fadd_rn(sum[c + j], __uint_as_float(r[j]));
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(acc ? tempty_leader1 : tempty_leader0);
                if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
            }
            if (stop) break;

            const int lrow = quarter * 32 + lane;
            const int lcol = cgroup * COLS;
            const int64_t row = (int64_t)w.tm * Cf::BM + (int64_t)rank * Cf::HM + lrow;
            const int64_t col0 = (int64_t)w.tn * BN + lcol;
            if (w.sti < 0) {
                if (cbuf) store_rows_tma<COLS>(&tmC, cbuf, sum, lane, row - lane, col0, M, N);
                else store_row_regs<COLS>(sum, p.C, row, col0, M, N, vec);
                continue;
            }
            // K-split tile: this CTA's 128-row half is its own partial tile.
            constexpr size_t TILE = (size_t)Cf::HM * BN;
            const int64_t half = w.sti * 2 + rank;
            finish_slice<COLS>(sum, p.partial + (size_t)half * p.max_splits * TILE + (size_t)lcol * 128 + lrow, TILE,
                               w.z, w.nsplit, p.reduce_after != 0, p.counters + (size_t)half * Cf::EPI + ew, lane, p.C,
                               row, col0, M, N, vec);
        }
        if (cbuf && lane == 0) bulk_wait_all();       // this warp's TMA stores have completed
    }

    tc_fence_before();
    __syncthreads();
    cluster_sync();                 // no CTA leaves while its peer may still touch it
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc_pair(tmem_base, Cf::TMEM_COLS);
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

// Raises a kernel's dynamic shared memory limit once per device (not inside
// a later stream capture).
template <typename Kern>
cudaError_t set_smem_once(Kern kern, int bytes, std::atomic<uint64_t>& done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// ============================================================================
// Fused-split variant (BF16x6 / BF16x9, 128 x 128 tiles). The operands are
// split inside the kernel instead of by the pre-pass. Warp 0 loads FP32 tiles
// of A (128 rows x 32 k) and B (32 k x 128 n, as four 32-column boxes) with
// TMA and the 128-byte swizzle into a staging ring, a few stages after an L2
// prefetch of the same boxes; eight converter warps cut each staged element
// into its three BF16 limbs (split_math.cuh, the pre-pass's arithmetic). A's
// limbs go to tensor memory, one row per TMEM lane, where the MMA reads them
// as its A operand; B's limb planes go to an operand ring in shared memory in
// the layout TMA writes for the pre-pass planes (128-byte column panels, the
// 128-byte swizzle). Keeping A out of shared memory takes its plane stores and
// the MMA's A reads (a third of the CTA's shared-memory traffic per stage) off
// the shared-memory pipe, which the MMA, TMA and the converters otherwise
// saturate on these 128-column tiles. The products, their order and the
// epilogue are those of the one-CTA kernel.
// Each FP32 element crosses HBM once per tile that reads it instead of being
// read, written as planes and read again: the gain where the pre-pass costs
// as much as the products (narrow M or N).
// ============================================================================
template <int MODE>
struct CfgFused {
    static constexpr int P = 3;                      // BF16 limb planes per operand
    static constexpr int ES = 2;
    static constexpr int BM = 128, BN = 128;
    static constexpr int BK = 32;                    // k per stage: one 64-byte row of BF16
    static constexpr int KSTEP = 16;
    static constexpr int KSTEPS = BK / KSTEP;
    static constexpr int B_PLANE = BK * BN * ES;     // 8 KB per B plane: 2 panels of 32 k x 128 bytes
    static constexpr int OP_STAGE = P * B_PLANE;     // B's limb planes; A's limbs are in TMEM
    static constexpr int OP_STAGES = 2;
    static constexpr int ST_A = BM * BK * 4;         // FP32 A box: 128 rows x 128 bytes
    static constexpr int ST_BOX = BK * 32 * 4;       // FP32 B box: 32 k x 32 n
    static constexpr int NBOX = BN / 32;
    static constexpr int ST_STAGE = ST_A + NBOX * ST_BOX;
    static constexpr int ST_STAGES = 5;
    static constexpr int PREFETCH = 6;               // stages between a box's L2 prefetch and its load
    static_assert(PREFETCH >= ST_STAGES, "prefetches run ahead of the staging ring");
    static constexpr int RING = OP_STAGES * OP_STAGE + ST_STAGES * ST_STAGE;
    static constexpr int NPROD = (MODE == MAXMULSK_PREC_BF16X6) ? 6 : 9;
    static constexpr uint32_t IDESC = make_idesc(1u, 128u, (uint32_t)BN, 1u);
    static constexpr int NACC = 2;                   // TMEM accumulators: columns 0 .. 255
    static constexpr uint32_t SUM_COL = NACC * BN;   // the unit's running sums: columns 256 .. 383
    static constexpr uint32_t A_COL = SUM_COL + BN;  // A's limbs: columns 384 .. 479
    static constexpr uint32_t A_SLOT = P * BK / 2;   // 48 columns per operand stage: limb p at 16 p
    static constexpr uint32_t TMEM_COLS = 512;
    static_assert(A_COL + OP_STAGES * A_SLOT <= TMEM_COLS, "TMEM columns");
    static constexpr int EPI = 4;                    // epilogue warps 2 .. 5, one per TMEM lane quarter
    static constexpr int NCONV = 8;                  // converter warps 6 .. 13: four for A, four for B
    static constexpr int THREADS = 64 + 32 * (EPI + NCONV);
    // C leaves from the TMEM sums 32 columns at a time through registers.
    static constexpr bool TMA_STORE = false;
    static constexpr int SMEM = RING + 1024;
    static_assert(SMEM <= kSmemCap, "shared memory");
    static_assert(NCONV * 16 == BM && NCONV == 2 * NBOX, "one converter lane per A row and per B box row");
};

// Units of a grouped launch: device tables of problems, units (heaviest
// first) and per-problem FP32 tensor maps.
struct GroupSrc {
    const TcGroupArgs& g;
    __device__ __forceinline__ int64_t units() const { return g.nunits; }
    // C of a grouped problem is written from registers.
    __device__ __forceinline__ const CUtensorMap* store_map(const UnitView&) const { return nullptr; }
    // The r-th unit of this CTA: the units are sorted heaviest first and dealt
    // in a snake order (forward in even rounds, backward in odd rounds), which
    // evens out the sums of unequal units across CTAs.
    __device__ __forceinline__ int64_t unit_of(int64_t r) const {
        return r * gridDim.x + ((r & 1) ? (gridDim.x - 1 - blockIdx.x) : blockIdx.x);
    }
    __device__ __forceinline__ void get(int64_t u, UnitView& v) const {
        const TcGroupUnit gu = g.units[u];
        const TcGroupProblem& P = g.probs[gu.problem];
        v.w.tm = gu.tm;
        v.w.tn = gu.tn;
        v.w.z = gu.z;
        v.w.nsplit = P.splits;
        v.w.kbeg = (int64_t)gu.z * P.kchunk;
        v.w.kend = min(P.K, v.w.kbeg + P.kchunk);
        v.w.sti = P.splits > 1 ? (int64_t)gu.tm * P.tiles_n + gu.tn : -1;
        v.problem = gu.problem;
        v.M = P.M; v.N = P.N; v.C = P.C; v.partial = P.partial; v.counters = P.counters;
        v.max_splits = P.splits; v.chunk_kb = P.chunk_kb; v.reduce_after = 0;
    }
    __device__ __forceinline__ const void* map_a(const UnitView& v, const void*) const {
        return static_cast<const char*>(g.maps) + 256 * (size_t)v.problem;
    }
    __device__ __forceinline__ const void* map_b(const UnitView& v, const void*) const {
        return static_cast<const char*>(g.maps) + 256 * (size_t)v.problem + 128;
    }
    __device__ __forceinline__ void acquire(const void* a, const void* b) const {
        tmap_acquire(a);
        tmap_acquire(b);
    }
};

// Epilogue of the fused-split kernel: four warps, one per TMEM lane quarter,
// each thread one row of the 128 x 128 tile. A unit's running sums live in
// TMEM columns SUM_COL .. SUM_COL + 127 rather than in registers, which
// leaves the register budget to the eight converter warps: per chunk, 32
// columns at a time, the chunk's accumulator and the running sum are loaded,
// added with round-to-nearest (the first chunk is copied), and the sum is
// stored back -- the same adds, in the same order, as the register
// epilogue's. A whole tile then leaves from TMEM 32 columns at a time; a K
// slice writes its partial row, and the last slice to arrive on this warp's
// counter sums every slice in slice order, 32 columns at a time.
template <class Cf, class Src>
__device__ __forceinline__ void epilogue_role_tsum(const Src& src, int* err, long long timeout, uint32_t tmem_base,
                                                   uint64_t* tfull_bar, uint64_t* tempty_bar, volatile int& abort_s,
                                                   int warp, int lane) {
    constexpr int BN = Cf::BN;
    constexpr int W = 32;                             // columns per TMEM load
    auto fail = [&]() {
        atomicOr(err, kErrTimeout);
        abort_s = 1;
    };
    auto kblocks = [&](const Unit& w) -> int64_t { return (w.kend - w.kbeg + Cf::BK - 1) / Cf::BK; };
    const int ew = warp - 2;                          // epilogue warp 0 .. EPI-1
    const int quarter = warp & 3;                     // TMEM lanes 32*quarter .. +31
    const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
    const uint32_t tsum = tmem_base + lanes + Cf::SUM_COL;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool stop = false;
    for (int64_t round = 0, u = src.unit_of(0); u < src.units() && !stop; u = src.unit_of(++round)) {
        UnitView v;
        src.get(u, v);
        const Unit& w = v.w;
        const int64_t M = v.M, N = v.N;
        const bool vec = (N % 4 == 0) && ((reinterpret_cast<uintptr_t>(v.C) & 15) == 0) &&
                         (v.partial == nullptr || (reinterpret_cast<uintptr_t>(v.partial) & 15) == 0);
        const int64_t nkb = kblocks(w);
        for (int64_t kb0 = 0; kb0 < nkb; kb0 += v.chunk_kb) {
            int bad = abort_s;
            if (!bad && lane == 0) {
                if (!mbar_wait_bounded(&tfull_bar[acc], acc_phase, timeout)) { fail(); bad = 1; }
            }
            bad = __shfl_sync(0xffffffffu, bad, 0);
            if (bad) { stop = true; break; }
            tc_fence_after();
            const uint32_t tacc = tmem_base + lanes + (uint32_t)(acc * BN);
#pragma unroll
            for (int c = 0; c < BN; c += W) {
                uint32_t r[W];
                tmem_ld_32x32b_x32(tacc + (uint32_t)c, r);
                if (kb0 == 0) {
                    tmem_wait_ld();
                    tmem_st_32x32b_x32(tsum + (uint32_t)c, r);
                } else {
                    uint32_t q[W];
                    tmem_ld_32x32b_x32(tsum + (uint32_t)c, q);
                    tmem_wait_ld();
#pragma unroll
                    for (int j = 0; j < W; j++)
                        q[j] = __float_as_uint(__fadd_rn(__uint_as_float(q[j]), __uint_as_float(r[j])));
                    tmem_st_32x32b_x32(tsum + (uint32_t)c, q);
                }
            }
            tmem_wait_st();                           // the sums are in TMEM before the next chunk reads them
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty_bar[acc]);
            if (++acc == Cf::NACC) { acc = 0; acc_phase ^= 1u; }
        }
        if (stop) break;

        // ---- the unit's sums are complete in TMEM: store them
        const int lrow = quarter * 32 + lane;         // row within the tile
        const int64_t row = (int64_t)w.tm * Cf::BM + lrow;
        const int64_t col0 = (int64_t)w.tn * BN;
        if (w.sti < 0) {
#pragma unroll
            for (int c = 0; c < BN; c += W) {
                uint32_t q[W];
                tmem_ld_32x32b_x32(tsum + (uint32_t)c, q);
                tmem_wait_ld();
                float f[W];
#pragma unroll
                for (int j = 0; j < W; j++) f[j] = __uint_as_float(q[j]);
                store_row_regs<W>(f, v.C, row, col0 + c, M, N, vec);
            }
            continue;
        }
        // Partial tiles column-major (element (r, c) at c * 128 + r): the 32
        // lanes of a warp hold 32 consecutive rows, so each store of one
        // column is one contiguous 128-byte line.
        constexpr size_t TILE = (size_t)Cf::BM * BN;
        float* seg = v.partial + (size_t)w.sti * v.max_splits * TILE + (size_t)lrow;
        float* part = seg + (size_t)w.z * TILE;
#pragma unroll
        for (int c = 0; c < BN; c += W) {
            uint32_t q[W];
            tmem_ld_32x32b_x32(tsum + (uint32_t)c, q);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < W; j++) __stcg(part + (size_t)(c + j) * Cf::BM, __uint_as_float(q[j]));
        }
        if (v.reduce_after) continue;
        unsigned* ctr = v.counters + (size_t)w.sti * Cf::EPI + ew;
        __threadfence();
        __syncwarp();
        int last = 0;
        if (lane == 0) last = (atomicAdd(ctr, 1u) == (unsigned)(w.nsplit - 1));
        last = __shfl_sync(0xffffffffu, last, 0);
        if (!last) continue;
        __threadfence();
#pragma unroll 1
        for (int c = 0; c < BN; c += W) {
            float sum[W];
#pragma unroll
            for (int j = 0; j < W; j++) sum[j] = __ldcg(seg + (size_t)(c + j) * Cf::BM);
            for (int qz = 1; qz < w.nsplit; qz++) {
                const float* bq = seg + (size_t)qz * TILE;
#pragma unroll
                for (int j = 0; j < W; j++) sum[j] = __fadd_rn(sum[j], __ldcg(bq + (size_t)(c + j) * Cf::BM));
            }
            store_row_regs<W>(sum, v.C, row, col0 + c, M, N, vec);
        }
        if (lane == 0) *ctr = 0u;
    }
}

template <int MODE, class Src>
__device__ __forceinline__ void fused_roles(const Src& src, const void* tmA1, const void* tmB1, const void* tmC1,
                                            int* err, long long timeout) {
    using Cf = CfgFused<MODE>;
    constexpr int BN = Cf::BN;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t st_full[Cf::ST_STAGES];
    __shared__ __align__(8) uint64_t st_empty[Cf::ST_STAGES];
    __shared__ __align__(8) uint64_t op_full[Cf::OP_STAGES];
    __shared__ __align__(8) uint64_t op_empty[Cf::OP_STAGES];
    __shared__ __align__(8) uint64_t tfull_bar[Cf::NACC];
    __shared__ __align__(8) uint64_t tempty_bar[Cf::NACC];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* ops = smem;                                        // operand ring (1024-aligned stages)
    uint8_t* stg = smem + Cf::OP_STAGES * Cf::OP_STAGE;         // staging ring
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    constexpr int CONV0 = 2 + Cf::EPI;                          // first converter warp

    if (threadIdx.x == 0) {
        for (int s = 0; s < Cf::ST_STAGES; s++) { mbar_init(&st_full[s], 1); mbar_init(&st_empty[s], Cf::NCONV); }
        for (int s = 0; s < Cf::OP_STAGES; s++) { mbar_init(&op_full[s], Cf::NCONV); mbar_init(&op_empty[s], 1); }
        for (int a = 0; a < Cf::NACC; a++) { mbar_init(&tfull_bar[a], 1); mbar_init(&tempty_bar[a], Cf::EPI); }
        mbar_init(&done_bar, 1);
        abort_s = 0;
        fence_mbar_init();
        fence_proxy_async();
    }
    if (warp == 0 && lane == 0 && tmA1) {
        prefetch_tmap(tmA1);
        prefetch_tmap(tmB1);
        if (tmC1) prefetch_tmap(tmC1);
    }
    if (warp == 1) { tmem_alloc(&tmem_base_s, Cf::TMEM_COLS); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = tmem_base_s;

    auto fail = [&]() {
        atomicOr(err, kErrTimeout);
        abort_s = 1;
    };
    auto kblocks = [&](const Unit& w) -> int64_t { return (w.kend - w.kbeg + Cf::BK - 1) / Cf::BK; };

    if (warp == 0) {
        // ------------------------------------------------------------ producer (FP32 tiles)
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t issued = 0;
            for (int64_t round = 0, u = src.unit_of(0); u < src.units() && !abort_s; u = src.unit_of(++round)) {
                UnitView v;
                src.get(u, v);
                const Unit& w = v.w;
                const void* mapA = src.map_a(v, tmA1);
                const void* mapB = src.map_b(v, tmB1);
                src.acquire(mapA, mapB);
                const int64_t nkb = kblocks(w);
                // The FP32 boxes of stage j go to L2 PREFETCH stages before
                // their load, which then waits for L2 instead of HBM. The
                // first stages are loaded at once (their loads go to HBM
                // themselves); each prefetch follows a load.
                auto prefetch = [&](int64_t j) {
                    const int32_t k = (int32_t)(w.kbeg + j * Cf::BK);
                    tma_prefetch_l2_2d(mapA, k, w.tm * Cf::BM);
#pragma unroll
                    for (int b = 0; b < Cf::NBOX; b++) tma_prefetch_l2_2d(mapB, w.tn * BN + 32 * b, k);
                };
                bool ok = true;
                for (int64_t kb = 0; kb < nkb; kb++) {
                    if (!mbar_wait_bounded(&st_empty[stage], phase ^ 1u, timeout)) { fail(); ok = false; break; }
                    if (abort_s) { ok = false; break; }
                    uint8_t* sa = stg + (size_t)stage * Cf::ST_STAGE;
                    mbar_arrive_expect_tx(&st_full[stage], (uint32_t)Cf::ST_STAGE);
                    const int32_t k = (int32_t)(w.kbeg + kb * Cf::BK);
                    tma_load_2d(sa, mapA, &st_full[stage], k, w.tm * Cf::BM);
#pragma unroll
                    for (int b = 0; b < Cf::NBOX; b++)
                        tma_load_2d(sa + Cf::ST_A + b * Cf::ST_BOX, mapB, &st_full[stage], w.tn * BN + 32 * b, k);
                    // Stages the ring does not hold yet: prefetched behind this load.
                    for (int64_t j = (kb == 0 ? Cf::ST_STAGES : kb + Cf::PREFETCH); j <= kb + Cf::PREFETCH && j < nkb; j++)
                        prefetch(j);
                    issued++;
                    if (++stage == Cf::ST_STAGES) { stage = 0; phase ^= 1u; }
                }
                if (!ok) break;
            }
            // No copy may still be landing in shared memory when the CTA exits.
            const int64_t first = issued > Cf::ST_STAGES ? issued - Cf::ST_STAGES : 0;
            for (int64_t j = first; j < issued; j++) {
                if (!mbar_wait_bounded(&st_full[j % Cf::ST_STAGES], (uint32_t)((j / Cf::ST_STAGES) & 1), timeout)) {
                    atomicOr(err, kErrTimeout);
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
            bool ok = true;
            for (int64_t round = 0, u = src.unit_of(0); u < src.units() && ok && !abort_s; u = src.unit_of(++round)) {
                UnitView v;
                src.get(u, v);
                const int64_t nkb = kblocks(v.w);
                for (int64_t kb0 = 0; kb0 < nkb && ok; kb0 += v.chunk_kb) {
                    if (!mbar_wait_bounded(&tempty_bar[acc], acc_phase ^ 1u, timeout)) { fail(); ok = false; break; }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                    const int64_t kb1 = min(nkb, kb0 + (int64_t)v.chunk_kb);
                    for (int64_t kb = kb0; kb < kb1; kb++) {
                        if (!mbar_wait_bounded(&op_full[stage], phase, timeout)) { fail(); ok = false; break; }
                        tc_fence_after();
                        const uint32_t a_tm = tmem_base + Cf::A_COL + (uint32_t)stage * Cf::A_SLOT;
                        const uint32_t b_base = smem_u32(ops + (size_t)stage * Cf::OP_STAGE);
#pragma unroll
                        for (int ks = 0; ks < Cf::KSTEPS; ks++) {
#pragma unroll
                            for (int q = 0; q < Cf::NPROD; q++) {
                                int pa, pb;
                                product_planes(MODE, q, pa, pb);
                                const uint32_t a_addr = a_tm + (uint32_t)(pa * (Cf::BK / 2) + ks * (Cf::KSTEP / 2));
                                const uint64_t bdesc =
                                    make_smem_desc(b_base + (uint32_t)(pb * Cf::B_PLANE + ks * Cf::KSTEP * 128),
                                                   (uint32_t)(Cf::BK * 128), 1024u, 2u);
                                const uint32_t accum = (kb > kb0 || ks > 0 || q > 0) ? 1u : 0u;
                                mma_bf16_ta(d_tmem, a_addr, bdesc, Cf::IDESC, accum);
                            }
                        }
                        tc_commit(&op_empty[stage]);
                        if (++stage == Cf::OP_STAGES) { stage = 0; phase ^= 1u; }
                    }
                    if (!ok) break;
                    tc_commit(&tfull_bar[acc]);
                    if (++acc == Cf::NACC) { acc = 0; acc_phase ^= 1u; }
                }
            }
            // No MMA may still be running when TMEM is freed.
            tc_commit(&done_bar);
            if (!mbar_wait_bounded(&done_bar, 0u, timeout)) { atomicOr(err, kErrTimeout); abort_s = 1; }
        }
    } else if (warp < CONV0) {
        // ------------------------------------------------------------ epilogue
        epilogue_role_tsum<Cf>(src, err, timeout, tmem_base, tfull_bar, tempty_bar, abort_s, warp, lane);
    } else {
        // ------------------------------------------------------------ converters
        // Warps cw = 0..3 split A rows 32q .. 32q+31 (one per lane), q = warp % 4
        // the TMEM lane quarter the warp may write; warps 4..7 split the 32 k
        // rows of B box cw - 4 (columns 32(cw-4) .. +31), one k row per lane:
        // two converter warps per SM sub-partition, so one warp's memory
        // traffic overlaps the other's arithmetic. Shared-memory accesses: a
        // quarter-warp covers 8 consecutive rows, whose swizzled 16-byte chunks
        // fall on distinct banks.
        const int cwx = warp - CONV0;
        const bool conv_a = cwx < Cf::NCONV / 2;
        const int cw = conv_a ? cwx : cwx - Cf::NCONV / 2;
        int stage = 0, ostage = 0;
        uint32_t phase = 0, ophase = 0;
        bool stop = false;
        for (int64_t round = 0, u = src.unit_of(0); u < src.units() && !stop; u = src.unit_of(++round)) {
            UnitView v;
            src.get(u, v);
            const int64_t nkb = kblocks(v.w);
            for (int64_t kb = 0; kb < nkb; kb++) {
                int bad = abort_s;
                if (!bad && lane == 0) {
                    if (!mbar_wait_bounded(&op_empty[ostage], ophase ^ 1u, timeout) ||
                        !mbar_wait_bounded(&st_full[stage], phase, timeout)) {
                        fail();
                        bad = 1;
                    }
                }
                bad = __shfl_sync(0xffffffffu, bad, 0);
                if (bad) { stop = true; break; }
                const uint8_t* sa = stg + (size_t)stage * Cf::ST_STAGE;
                uint8_t* oa = ops + (size_t)ostage * Cf::OP_STAGE;
                if (conv_a) {
                    // A row r: 32 FP32 k's (128-byte row, 128-byte swizzle) ->
                    // three limbs of 16 packed k pairs, stored in TMEM lane r at
                    // columns A_COL + A_SLOT ostage + 16 p + pair.
                    const int quarter = warp & 3;
                    const int r = quarter * 32 + lane;
                    float x[32];
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const float4 v = *reinterpret_cast<const float4*>(sa + r * 128 + ((c ^ (r & 7)) << 4));
                        x[4 * c] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
                    }
                    // The MMAs that read this slot (two stages back) are done.
                    tc_fence_after();
                    const uint32_t ta = tmem_base + ((uint32_t)(quarter * 32) << 16) + Cf::A_COL +
                                        (uint32_t)ostage * Cf::A_SLOT;
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        uint32_t l0[8], l1[8], l2[8];
#pragma unroll
                        for (int e = 0; e < 8; e++)
                            bf16_limbs2(x[16 * h + 2 * e], x[16 * h + 2 * e + 1], l0[e], l1[e], l2[e]);
                        tmem_st_32x32b_x8(ta + (uint32_t)(8 * h), l0);
                        tmem_st_32x32b_x8(ta + (uint32_t)(16 + 8 * h), l1);
                        tmem_st_32x32b_x8(ta + (uint32_t)(32 + 8 * h), l2);
                    }
                    // The limbs are in TMEM before the MMA warp is told.
                    tmem_wait_st();
                    tc_fence_before();
                } else {
                    // B row k of box cw: 32 FP32 n's -> four 16-byte chunks of
                    // 8 BF16 in column panel cw / 2, chunks 4 (cw % 2) .. +3.
                    const int k = lane;
                    const uint8_t* sb = sa + Cf::ST_A + cw * Cf::ST_BOX;
                    float x[32];
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const float4 v = *reinterpret_cast<const float4*>(sb + k * 128 + ((c ^ (k & 7)) << 4));
                        x[4 * c] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
                    }
                    uint8_t* ob = oa + (cw >> 1) * (Cf::BK * 128) + k * 128;
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        uint32_t l0[4], l1[4], l2[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) bf16_limbs2(x[8 * j + 2 * e], x[8 * j + 2 * e + 1], l0[e], l1[e], l2[e]);
                        const int off = ((((cw & 1) * 4 + j) ^ (k & 7)) << 4);
                        *reinterpret_cast<uint4*>(ob + off) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
                        *reinterpret_cast<uint4*>(ob + Cf::B_PLANE + off) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
                        *reinterpret_cast<uint4*>(ob + 2 * Cf::B_PLANE + off) = make_uint4(l2[0], l2[1], l2[2], l2[3]);
                    }
                    // The planes are read by the tensor cores (async proxy).
                    fence_proxy_async();
                }
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&op_full[ostage]);
                    mbar_arrive(&st_empty[stage]);
                }
                if (++stage == Cf::ST_STAGES) { stage = 0; phase ^= 1u; }
                if (++ostage == Cf::OP_STAGES) { ostage = 0; ophase ^= 1u; }
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

template <int MODE, bool GROUPED>
__global__ void __launch_bounds__(CfgFused<MODE>::THREADS, 1)
tc_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmC, const TcParams p, const TcGroupArgs g) {
    if constexpr (GROUPED) {
        fused_roles<MODE>(GroupSrc{g}, nullptr, nullptr, nullptr, g.err, g.timeout);
    } else {
        const CUtensorMap* c = p.store_c ? &tmC : nullptr;
        fused_roles<MODE>(SingleSrc{p, c}, &tmA, &tmB, c, p.err, p.timeout);
    }
}

// Split-K reduction for plans that cut every tile into K slices. The GEMM
// wrote one partial tile per (128-row half, slice); each thread here sums one
// element over the slices in slice order -- the order of the in-kernel fixup,
// so C is the same bit for bit -- and stores it. The slices of a tile are
// read by many threads at once, 16 loads in flight per thread, instead of one
// warp walking them in turn at the end of the GEMM. HBM-bound: nsplit
// partials in, C out.
template <int BN>
__global__ void __launch_bounds__(256)
tc_splitk_reduce_kernel(const TcParams p) {
    constexpr size_t TILE = (size_t)128 * BN;
    const int halves = p.bm / 128;
    const int64_t total = p.tiles * halves * (int64_t)TILE;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        // Partial tiles are column-major (c * 128 + r): consecutive threads
        // read consecutive partial elements down a column.
        const int lrow = (int)(i % 128);
        const int q = (int)((i / 128) % BN);
        const int64_t th = i / (int64_t)TILE;                   // tile * halves + half
        const int64_t t = halves == 2 ? th >> 1 : th;
        int tm, tn;
        if (p.tiles <= (int64_t)UINT32_MAX) tile_coords_t<uint32_t>(p, (uint32_t)t, tm, tn);
        else tile_coords_t<uint64_t>(p, (uint64_t)t, tm, tn);
        const int64_t row = (int64_t)tm * p.bm + (th - t * halves) * 128 + lrow;
        const int64_t col = (int64_t)tn * BN + q;
        if (row >= p.M || col >= p.N) continue;
        const float* src = p.partial + (size_t)th * p.max_splits * TILE + (size_t)q * 128 + (size_t)lrow;
        p.C[(size_t)row * (size_t)p.N + (size_t)col] = ordered_sum(src, TILE, p.main_splits);
    }
}

// A K split of every tile into at least this many slices is summed by
// tc_splitk_reduce_kernel; fewer slices (and tail-wave splits) by the last
// slice to arrive, inside the GEMM.
constexpr int kReduceAfterSplits = 3;

template <int BN>
cudaError_t launch_reduce(const TcParams& prm, cudaStream_t s) {
    const int64_t total = prm.tiles * (prm.bm / 128) * 128 * BN;
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)device_sm_count() * 8;
    if (cap > 0 && blocks > cap) blocks = cap;
    tc_splitk_reduce_kernel<BN><<<(unsigned)blocks, 256, 0, s>>>(prm);
    return cudaGetLastError();
}

// Host-side schedule of one launch (see TcParams).
struct Sched {
    int bm;                          // rows per tile (128, or 256 for CTA pairs)
    int64_t tiles_m, tiles_n, tiles;
    int64_t main_tiles, main_units, units;
    int main_splits, tail_splits;
    int64_t main_kchunk, tail_kchunk;
    int64_t split_tiles;
    int max_splits;
    int64_t grid;
};

// With no K split requested and a last wave that would leave SMs idle
// (tiles = w * SMs + r, 0 < r <= SMs / 2), the r tiles of that wave are cut
// into floor(SMs / r) K slices so the wave is shared by all SMs.
Sched make_sched(int64_t M, int64_t K, int64_t N, int tile_m, int tile_n, int split_k, int slots) {
    int sms = slots;
    Sched s{};
    s.bm = tile_m;
    s.tiles_m = (M + tile_m - 1) / tile_m;
    s.tiles_n = (N + tile_n - 1) / tile_n;
    s.tiles = s.tiles_m * s.tiles_n;
    if (sms <= 0) sms = 148;                        // work slots: SMs, or resident CTA pairs
    if (split_k == 0) {
        // Fill the machine: every tile cut into as many K slices as there are
        // slots per tile, so the units number about one per slot and each runs
        // the same number of k-steps (a stream-K schedule in whole slices).
        const int64_t f = sms / s.tiles;
        split_k = (int)(f < 1 ? 1 : (f > 64 ? 64 : f));
    }
    s.main_splits = slice_count((size_t)K, split_k);
    s.main_kchunk = (int64_t)slice_len((size_t)K, split_k);
    s.main_tiles = s.tiles;
    s.tail_splits = 1;
    s.tail_kchunk = K;
    if (s.main_splits == 1 && s.tiles > sms) {
        const int64_t r = s.tiles % sms;
        if (r > 0 && r <= sms / 2) {
            int want = (int)(sms / r);
            const int64_t max_by_k = K / 256;          // keep slices at least 256 deep
            if (want > max_by_k) want = (int)max_by_k;
            if (want > 1) {
                const int tail = slice_count((size_t)K, want);
                if (tail > 1) {
                    s.tail_splits = tail;
                    s.tail_kchunk = (int64_t)slice_len((size_t)K, want);
                    s.main_tiles = s.tiles - r;
                }
            }
        }
    }
    s.main_units = s.main_tiles * s.main_splits;
    s.units = s.main_units + (s.tiles - s.main_tiles) * s.tail_splits;
    if (s.main_splits > 1) { s.split_tiles = s.tiles; s.max_splits = s.main_splits; }
    else if (s.tail_splits > 1) { s.split_tiles = s.tiles - s.main_tiles; s.max_splits = s.tail_splits; }
    else { s.split_tiles = 0; s.max_splits = 1; }
    s.grid = s.units < sms ? s.units : sms;
    return s;
}

// K per TMEM accumulation chunk. Measured on B200: the split product's
// normwise error grows with the chunk (at 4096^3, U[-1,1): 0.31x / 0.47x /
// 0.84x / 1.6x the plain FP32 kernel's for 32 / 64 / 128 / 256; wide exponent
// ranges about 1.65x more, relative), and falls with K relative to the plain
// kernel, whose single chain lengthens with K (128 x 32768 x 512, N(0, 1/K):
// 0.53x at 256). Each chunk costs one TMEM drain: at 4096^3 the CTA-pair
// GEMM ran 592 us with chunks of 64 and 507 us with 256, and narrow K-split
// plans 13 % faster with 256 than with 32. Tiers by K that keep every
// benchmark cell within the 2x bar with room: 32 below K = 4096, 128 below
// 16384, 256 above; a K-split plan takes the tier of its whole K (its chains
// are no longer than an unsplit plan's).
int chunk_len(int64_t K, int splits) {
    (void)splits;
    if (K >= 16384) return 256;
    if (K >= 4096) return 128;
    return 32;
}

// Split tiles keep one partial per 128-row half (a CTA's rows) and slice, and
// one arrival counter per half and epilogue warp.
size_t counter_bytes(const Sched& s) {
    return (size_t)s.split_tiles * (s.bm / 128) * 8 * sizeof(unsigned);
}
size_t partial_bytes(const Sched& s, int tile_n) {
    if (s.split_tiles == 0) return 0;
    return align256(counter_bytes(s)) +
           align256((size_t)s.split_tiles * (s.bm / 128) * s.max_splits * 128 * (size_t)tile_n * sizeof(float));
}

// Kernel parameters of one launch: the problem, its schedule, and the K per
// stage of the configuration (for the TMEM chunk length in stages).
TcParams make_params(const TcArgs& a, const Sched& sc, int bk) {
    TcParams prm;
    prm.M = a.M; prm.K = a.K; prm.N = a.N;
    prm.bm = sc.bm;
    prm.tiles_m = (int)sc.tiles_m;
    prm.tiles_n = (int)sc.tiles_n;
    prm.tiles = sc.tiles;
    prm.main_tiles = sc.main_tiles;
    prm.main_units = sc.main_units;
    prm.units = sc.units;
    prm.main_splits = sc.main_splits;
    prm.tail_splits = sc.tail_splits;
    prm.main_kchunk = sc.main_kchunk;
    prm.tail_kchunk = sc.tail_kchunk;
    prm.max_splits = sc.max_splits;
    prm.chunk_kb = (a.chunk > 0 ? a.chunk : chunk_len(a.K, sc.main_splits)) / bk;
    prm.reduce_after = (sc.main_splits >= kReduceAfterSplits) ? 1 : 0;
    prm.store_c = 0;
    prm.C = a.C;
    prm.partial = a.partial;
    prm.counters = a.counters;
    prm.err = a.err;
    prm.timeout = 2000000000LL;   // about one second at B200 clocks
    return prm;
}

// C as the TMA-store writeback sees it: M rows of N FP32, boxes of 32 x 32
// with the 128-byte swizzle. Needs rows of a multiple of 16 bytes, a 16-byte
// aligned C and 32-bit box coordinates; otherwise (false) whole tiles are
// stored from registers.
bool encode_c_map(float* C, int64_t M, int64_t N, CUtensorMap* tm) {
    std::memset(tm, 0, sizeof *tm);
    EncodeTiledFn enc = get_encode_fn();
    if (!enc || M <= 0 || N <= 0 || M > INT32_MAX || N > INT32_MAX || N % 4 != 0 ||
        (reinterpret_cast<uintptr_t>(C) & 15) != 0)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)M};
    const cuuint64_t strides[1] = {(cuuint64_t)N * 4u};
    const cuuint32_t box[2] = {(cuuint32_t)kStoreBox, 32u};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        std::memset(tm, 0, sizeof *tm);
        return false;
    }
    return true;
}

template <int MODE, int BN>
cudaError_t launch_cfg(const TcArgs& a, cudaStream_t s) {
    using Cf = Cfg<MODE, BN>;
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const PlaneGeom g = plane_geom(a.M, a.K, a.N, a.precision);
    char* a_planes = static_cast<char*>(a.planes);
    char* b_planes = a.b_planes ? static_cast<char*>(a.b_planes) : a_planes + (size_t)g.P * g.a_plane_bytes;
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
    if constexpr (Cf::B_KMAJOR) {
        const cuuint64_t dims[3] = {(cuuint64_t)g.Kp, (cuuint64_t)a.N, (cuuint64_t)g.P};
        const cuuint64_t strides[2] = {(cuuint64_t)g.Kp * Cf::ES, (cuuint64_t)g.b_plane_bytes};
        const cuuint32_t box[3] = {(cuuint32_t)Cf::BK, (cuuint32_t)BN, (cuuint32_t)Cf::P};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&tmB, dt, 3, b_planes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    } else {
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

    const Sched sc = make_sched(a.M, a.K, a.N, 128, BN, a.split_k, tc_slots(a.precision, 128, BN));
    TcParams prm = make_params(a, sc, Cf::BK);
    if (sc.split_tiles > 0 && (!a.partial || !a.counters)) return cudaErrorInvalidValue;
    CUtensorMap tmC;
    prm.store_c = (encode_c_map(a.C, a.M, a.N, &tmC) && Cf::TMA_STORE) ? 1 : 0;

    static std::atomic<uint64_t> smem_set{0};
    cudaError_t e = set_smem_once(tc_gemm_kernel<MODE, BN>, Cf::SMEM, smem_set);
    if (e != cudaSuccess) return e;
    {
        PhaseScope ps(kPhaseGemm, s);
        tc_gemm_kernel<MODE, BN><<<(unsigned)sc.grid, Cf::THREADS, Cf::SMEM, s>>>(tmA, tmB, tmC, prm);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess || !prm.reduce_after) return e;
    PhaseScope ps(kPhaseReduce, s);
    return launch_reduce<BN>(prm, s);
}

template <int MODE, int BN>
cudaError_t launch_cfg_pair(const TcArgs& a, cudaStream_t s) {
    using Cf = CfgPair<MODE, BN>;
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const PlaneGeom g = plane_geom(a.M, a.K, a.N, a.precision);
    char* a_planes = static_cast<char*>(a.planes);
    char* b_planes = a.b_planes ? static_cast<char*>(a.b_planes) : a_planes + (size_t)g.P * g.a_plane_bytes;
    const CUtensorMapDataType dt = Cf::TF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;

    CUtensorMap tmA, tmB;
    {
        const cuuint64_t dims[3] = {(cuuint64_t)g.Kp, (cuuint64_t)a.M, (cuuint64_t)g.P};
        const cuuint64_t strides[2] = {(cuuint64_t)g.Kp * Cf::ES, (cuuint64_t)g.a_plane_bytes};
        const cuuint32_t box[3] = {(cuuint32_t)Cf::BK, (cuuint32_t)Cf::HM, (cuuint32_t)Cf::P};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&tmA, dt, 3, a_planes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    if constexpr (Cf::B_KMAJOR) {
        const cuuint64_t dims[3] = {(cuuint64_t)g.Kp, (cuuint64_t)a.N, (cuuint64_t)g.P};
        const cuuint64_t strides[2] = {(cuuint64_t)g.Kp * Cf::ES, (cuuint64_t)g.b_plane_bytes};
        const cuuint32_t box[3] = {(cuuint32_t)Cf::BK, (cuuint32_t)Cf::HN, (cuuint32_t)Cf::P};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&tmB, dt, 3, b_planes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    } else {
        const cuuint64_t npan = (cuuint64_t)(g.Np / Cf::NBE);
        const cuuint64_t dims[4] = {(cuuint64_t)Cf::NBE, (cuuint64_t)a.K, npan, (cuuint64_t)g.P};
        const cuuint64_t strides[3] = {128u, (cuuint64_t)a.K * 128u, (cuuint64_t)g.b_plane_bytes};
        const cuuint32_t box[4] = {(cuuint32_t)Cf::NBE, (cuuint32_t)Cf::BK, (cuuint32_t)Cf::HNBLK, (cuuint32_t)Cf::P};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        if (enc(&tmB, dt, 4, b_planes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }

    const Sched sc = make_sched(a.M, a.K, a.N, 256, BN, a.split_k, tc_slots(a.precision, 256, BN));
    TcParams prm = make_params(a, sc, Cf::BK);
    if (sc.split_tiles > 0 && (!a.partial || !a.counters)) return cudaErrorInvalidValue;
    CUtensorMap tmC;
    prm.store_c = (encode_c_map(a.C, a.M, a.N, &tmC) && Cf::TMA_STORE) ? 1 : 0;

    static std::atomic<uint64_t> smem_set{0};
    cudaError_t e = set_smem_once(tc_gemm_pair_kernel<MODE, BN>, Cf::SMEM, smem_set);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * sc.grid), 1, 1);
    cfg.blockDim = dim3(Cf::THREADS, 1, 1);
    cfg.dynamicSmemBytes = Cf::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    {
        PhaseScope ps(kPhaseGemm, s);
        e = cudaLaunchKernelEx(&cfg, tc_gemm_pair_kernel<MODE, BN>, tmA, tmB, tmC, prm);
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e != cudaSuccess || !prm.reduce_after) return e;
    PhaseScope ps(kPhaseReduce, s);
    return launch_reduce<BN>(prm, s);
}

// The fused-split kernel reads the FP32 operands directly: A as K x M rows of
// 4-byte elements, B as N x K; both need rows of a multiple of 16 bytes and a
// 16-byte aligned start (checked by the caller).
bool encode_fused_maps(const float* A, int64_t lda, const float* B, int64_t M, int64_t K, int64_t N,
                       CUtensorMap* tmA, CUtensorMap* tmB) {
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return false;
    constexpr int BK = CfgFused<MAXMULSK_PREC_BF16X6>::BK;
    constexpr int BM = CfgFused<MAXMULSK_PREC_BF16X6>::BM;
    const cuuint32_t estr[2] = {1, 1};
    {
        const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)M};
        const cuuint64_t strides[1] = {(cuuint64_t)lda * 4u};
        const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)BM};
        if (enc(tmA, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(A), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    {
        const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)K};
        const cuuint64_t strides[1] = {(cuuint64_t)N * 4u};
        const cuuint32_t box[2] = {32u, (cuuint32_t)BK};
        if (enc(tmB, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(B), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

template <int MODE>
cudaError_t launch_fused(const TcArgs& a, cudaStream_t s) {
    using Cf = CfgFused<MODE>;
    constexpr int BN = Cf::BN;
    CUtensorMap tmA, tmB;
    if (!encode_fused_maps(a.A, a.K, a.B, a.M, a.K, a.N, &tmA, &tmB)) return cudaErrorInvalidValue;
    const Sched sc = make_sched(a.M, a.K, a.N, 128, BN, a.split_k, tc_slots(a.precision, 128, BN));
    TcParams prm = make_params(a, sc, Cf::BK);
    if (sc.split_tiles > 0 && (!a.partial || !a.counters)) return cudaErrorInvalidValue;
    CUtensorMap tmC;
    prm.store_c = (encode_c_map(a.C, a.M, a.N, &tmC) && Cf::TMA_STORE) ? 1 : 0;

    static std::atomic<uint64_t> smem_set{0};
    cudaError_t e = set_smem_once(tc_fused_kernel<MODE, false>, Cf::SMEM, smem_set);
    if (e != cudaSuccess) return e;
    TcGroupArgs none{};
    {
        PhaseScope ps(kPhaseGemm, s);
        tc_fused_kernel<MODE, false><<<(unsigned)sc.grid, Cf::THREADS, Cf::SMEM, s>>>(tmA, tmB, tmC, prm, none);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess || !prm.reduce_after) return e;
    PhaseScope ps(kPhaseReduce, s);
    return launch_reduce<BN>(prm, s);
}

template <int MODE>
cudaError_t launch_mode(const TcArgs& a, cudaStream_t s) {
    if (a.tile_m == 256) {
        switch (a.tile_n) {
            case 128: return launch_cfg_pair<MODE, 128>(a, s);
            case 256: return launch_cfg_pair<MODE, 256>(a, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (a.tile_n) {
        case 64: return launch_cfg<MODE, 64>(a, s);
        case 128: return launch_cfg<MODE, 128>(a, s);
        case 256: return launch_cfg<MODE, 256>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int MODE, int BN>
int pair_slots_for() {
    using Cf = CfgPair<MODE, BN>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2, 1, 1);
    cfg.blockDim = dim3(Cf::THREADS, 1, 1);
    cfg.dynamicSmemBytes = Cf::SMEM;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaFuncSetAttribute(tc_gemm_pair_kernel<MODE, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Cf::SMEM) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, tc_gemm_pair_kernel<MODE, BN>, &cfg) != cudaSuccess) return 0;
    return n;
}

}  // namespace

// Concurrently resident work slots of a configuration on the current device:
// the SM count for one-CTA tiles, the number of CTA pairs that fit at once
// for 256-row tiles (cached per device and configuration).
int tc_slots(int precision, int tile_m, int tile_n) {
    if (tile_m != 256) return device_sm_count();
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_tuple(dev, precision, tile_n);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (precision == MAXMULSK_PREC_3XTF32) n = tile_n == 256 ? pair_slots_for<MAXMULSK_PREC_3XTF32, 256>()
                                                            : pair_slots_for<MAXMULSK_PREC_3XTF32, 128>();
    else if (precision == MAXMULSK_PREC_BF16X6) n = tile_n == 256 ? pair_slots_for<MAXMULSK_PREC_BF16X6, 256>()
                                                                 : pair_slots_for<MAXMULSK_PREC_BF16X6, 128>();
    else n = tile_n == 256 ? pair_slots_for<MAXMULSK_PREC_BF16X9, 256>() : pair_slots_for<MAXMULSK_PREC_BF16X9, 128>();
    if (n <= 0) n = device_sm_count() / 2;
    cache[key] = n;
    return n;
}

size_t tc_workspace_bytes(int64_t M, int64_t K, int64_t N, int precision, int tile_m, int tile_n, int split_k) {
    const PlaneGeom g = plane_geom(M, K, N, precision);
    const Sched sc = make_sched(M, K, N, tile_m, tile_n, split_k, tc_slots(precision, tile_m, tile_n));
    return align256((size_t)g.P * (g.a_plane_bytes + g.b_plane_bytes)) + partial_bytes(sc, tile_n);
}

// Counter bytes to clear before a launch: none when tc_splitk_reduce_kernel
// sums the slices (no counter is read), which saves a launch on K-split plans.
size_t tc_counter_bytes(int64_t M, int64_t K, int64_t N, int precision, int tile_m, int tile_n, int split_k) {
    const Sched sc = make_sched(M, K, N, tile_m, tile_n, split_k, tc_slots(precision, tile_m, tile_n));
    return sc.main_splits >= kReduceAfterSplits ? 0 : counter_bytes(sc);
}

bool tc_bind_workspace(TcArgs& a, void* ws, size_t ws_bytes) {
    const PlaneGeom g = plane_geom(a.M, a.K, a.N, a.precision);
    const Sched sc = make_sched(a.M, a.K, a.N, a.tile_m, a.tile_n, a.split_k,
                                tc_slots(a.precision, a.tile_m, a.tile_n));
    const size_t planes = align256((size_t)g.P * (g.a_plane_bytes + g.b_plane_bytes));
    const size_t need = planes + partial_bytes(sc, a.tile_n);
    if (!ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(ws) & 255) != 0) return false;
    char* base = static_cast<char*>(ws);
    a.planes = base;
    if (sc.split_tiles > 0) {
        a.counters = reinterpret_cast<unsigned*>(base + planes);
        a.partial = reinterpret_cast<float*>(base + planes + align256(counter_bytes(sc)));
    } else {
        a.counters = nullptr;
        a.partial = nullptr;
    }
    return true;
}

cudaError_t tc_launch(const TcArgs& a, cudaStream_t s) {
    if (a.fused) {
        if (a.tile_m != 128 || a.tile_n != 128) return cudaErrorInvalidValue;
        if (a.precision == MAXMULSK_PREC_BF16X6) return launch_fused<MAXMULSK_PREC_BF16X6>(a, s);
        if (a.precision == MAXMULSK_PREC_BF16X9) return launch_fused<MAXMULSK_PREC_BF16X9>(a, s);
        return cudaErrorInvalidValue;
    }
    if (!a.reuse_planes) {
        // With B's planes supplied from outside only A is split here.
        PhaseScope ps(kPhaseSplit, s);
        cudaError_t e = a.b_planes ? split_one(a.A, a.M, a.K, a.precision, false, a.planes, s)
                                   : split_launch(a.A, a.B, a.M, a.K, a.N, a.precision, a.planes, s);
        if (e != cudaSuccess) return e;
    }
    switch (a.precision) {
        case MAXMULSK_PREC_3XTF32: return launch_mode<MAXMULSK_PREC_3XTF32>(a, s);
        case MAXMULSK_PREC_BF16X6: return launch_mode<MAXMULSK_PREC_BF16X6>(a, s);
        case MAXMULSK_PREC_BF16X9: return launch_mode<MAXMULSK_PREC_BF16X9>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

bool tc_fused_maps(const float* A, int64_t lda, const float* B, int64_t M, int64_t K, int64_t N, void* out) {
    CUtensorMap* m = static_cast<CUtensorMap*>(out);
    return encode_fused_maps(A, lda, B, M, K, N, &m[0], &m[1]);
}

int tc_chunk_len(int64_t K, int splits) { return chunk_len(K, splits); }

cudaError_t tc_grouped_launch(const TcGroupArgs& g, int precision, int grid, cudaStream_t s) {
    static_assert(sizeof(CUtensorMap) == 128, "grouped tensor-map table stride");
    if (g.nunits <= 0) return cudaSuccess;
    CUtensorMap none{};
    const TcParams p{};
    if (precision == MAXMULSK_PREC_BF16X6) {
        using Cf = CfgFused<MAXMULSK_PREC_BF16X6>;
        static std::atomic<uint64_t> smem_set{0};
        cudaError_t e = set_smem_once(tc_fused_kernel<MAXMULSK_PREC_BF16X6, true>, Cf::SMEM, smem_set);
        if (e != cudaSuccess) return e;
        tc_fused_kernel<MAXMULSK_PREC_BF16X6, true><<<(unsigned)grid, Cf::THREADS, Cf::SMEM, s>>>(none, none, none, p, g);
    } else if (precision == MAXMULSK_PREC_BF16X9) {
        using Cf = CfgFused<MAXMULSK_PREC_BF16X9>;
        static std::atomic<uint64_t> smem_set{0};
        cudaError_t e = set_smem_once(tc_fused_kernel<MAXMULSK_PREC_BF16X9, true>, Cf::SMEM, smem_set);
        if (e != cudaSuccess) return e;
        tc_fused_kernel<MAXMULSK_PREC_BF16X9, true><<<(unsigned)grid, Cf::THREADS, Cf::SMEM, s>>>(none, none, none, p, g);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

namespace {
// One thread waits, with the kernels' bounded wait, on an mbarrier that no
// one arrives at; when the limit runs out it records the timeout in the device
// error word as the GEMM kernels do, and the kernel returns.
__global__ void timeout_probe_kernel(int* err, long long limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        if (!mbar_wait_bounded(&bar, 0u, limit)) atomicOr(err, kErrTimeout);
    }
}
}  // namespace

cudaError_t tc_timeout_probe(int* err, long long limit, cudaStream_t s) {
    timeout_probe_kernel<<<1, 32, 0, s>>>(err, limit);
    return cudaGetLastError();
}

}  // namespace mmsk
