// Internal declarations shared by the host runtime and the kernel files.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "maxmulsk.h"

namespace mmsk {

// K is cut into slices of kchunk elements; kchunk is a multiple of this so a
// slice boundary never splits a staging block of any kernel.
constexpr int kSliceAlign = 32;

// Slice length for a plan's split_k. The number of slices actually run is
// ceil(K / kchunk) <= split_k, so no slice is ever empty.
inline size_t slice_len(size_t K, int split_k) {
    if (split_k <= 1 || K == 0) return K;
    size_t per = (K + (size_t)split_k - 1) / (size_t)split_k;
    per = (per + kSliceAlign - 1) / kSliceAlign * kSliceAlign;
    return per < K ? per : K;
}
inline int slice_count(size_t K, int split_k) {
    size_t kc = slice_len(K, split_k);
    return kc ? (int)((K + kc - 1) / kc) : 1;
}

// Device-side error word bits (one int per device, see runtime.cpp).
enum : int {
    kErrTimeout = 1,
};

// ---------------------------------------------------------------------------
// SIMT FP32 kernels (simt.cu)
// ---------------------------------------------------------------------------
struct SimtArgs {
    const float* A; const float* B; float* C;
    int64_t M, K, N;
    int64_t kchunk;        // slice length (multiple of kSliceAlign) or K
    int splits;            // slices actually run (>= 1)
    float* partial;        // splits * M * N floats when splits > 1
    unsigned* counters;    // one per output tile when splits > 1 (zero on entry)
    int reduce_after;      // set by simt_launch: slices only write partials, a
                           // separate kernel sums them (zero everywhere else)
};
// Workspace bytes for the SIMT path with this tile/split choice.
size_t simt_workspace_bytes(int64_t M, int64_t K, int64_t N, int tile_m, int tile_n, int split_k);
// Lays out ws into SimtArgs fields. Returns false if ws is too small.
bool simt_bind_workspace(SimtArgs& a, int tile_m, int tile_n, void* ws, size_t ws_bytes);
cudaError_t simt_launch(const SimtArgs& a, int tile_m, int tile_n, int variant, cudaStream_t s);
// Grouped launch (one persistent kernel over many problems).
struct GroupProblem {
    SimtArgs a;            // one problem: pointers, sizes, its K slicing and scratch
    int32_t tiles_n;       // tiles along N (numbers the split-K counters)
    int32_t vec;           // 128-bit loads allowed for this problem
};
struct GroupUnit {
    int32_t problem, tm, tn, z;
};
cudaError_t simt_grouped_launch(const GroupProblem* probs, const GroupUnit* units, int nunits, unsigned* next,
                                int tile_m, int tile_n, int variant, int grid, cudaStream_t s);
// Runs an FP32 plan whose split-K scratch (counters, then partials) is at
// `scratch` (>= simt_workspace_bytes; may be null without a K split): lays it
// out, clears the counters on `s`, launches. Both the workspace entry and the
// static-scratch entry go through here.
maxmulsk_status simt_run(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                         const maxmulsk_plan& plan, void* scratch, size_t scratch_bytes, cudaStream_t s);
// The SIMT plan with its split-K scratch in a static device array (no allocation).
maxmulsk_status simt_run_static_scratch(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                        const maxmulsk_plan& plan, cudaStream_t s);

// ---------------------------------------------------------------------------
// Split-precision tensor-core path (split.cu, tc.cu)
// ---------------------------------------------------------------------------
struct TcArgs {
    const float* A; const float* B; float* C;
    int64_t M, K, N;
    int precision;         // MAXMULSK_PREC_3XTF32 / _BF16X6 / _BF16X9
    int tile_m;            // 128 (one CTA per tile) or 256 (a CTA pair per tile)
    int tile_n;            // 64, 128 or 256
    int split_k;           // the plan's split_k
    int chunk;             // k's per TMEM accumulation, 0 = chunk_len's choice
    bool reuse_planes;     // skip the split pre-pass: planes are already in place
    bool fused;            // split inside the GEMM kernel (BF16 modes, 128 x 128 tiles)
    void* planes;          // operand planes written by the split pre-pass
    void* b_planes;        // B's planes split earlier (split_one as_b), or null:
                           // then they follow A's planes in `planes`
    float* partial;        // compact partial tiles of the K-split tiles
    unsigned* counters;    // per split tile and epilogue warp (zero on entry)
    int* err;              // device error word
};
size_t tc_workspace_bytes(int64_t M, int64_t K, int64_t N, int precision, int tile_m, int tile_n, int split_k);
// Bytes of the arrival counters at the start of the partial area to zero
// before a launch (0 when the plan's slices are summed by a reduce kernel).
size_t tc_counter_bytes(int64_t M, int64_t K, int64_t N, int precision, int tile_m, int tile_n, int split_k);
// Concurrently resident work slots (SMs, or CTA pairs for 256-row tiles).
int tc_slots(int precision, int tile_m, int tile_n);
bool tc_bind_workspace(TcArgs& a, void* ws, size_t ws_bytes);
cudaError_t tc_launch(const TcArgs& a, cudaStream_t s);

// Grouped split-precision launch (fused split kernel over many GEMMs).
struct TcGroupProblem {
    int64_t M, K, N;
    float* C;
    float* partial;        // split problems: [tile][slice][128 x 128] floats
    unsigned* counters;    // split problems: 8 per tile (zero on entry)
    int64_t kchunk;        // K slice length
    int32_t tiles_n;       // tiles along N
    int32_t splits;        // K slices (1 = whole)
    int32_t chunk_kb;      // stages per TMEM accumulation chunk
    int32_t pad;
};
struct TcGroupUnit {
    int32_t problem, tm, tn, z;
};
struct TcGroupArgs {
    const TcGroupProblem* probs;
    const TcGroupUnit* units;
    const void* maps;      // per problem two 128-byte CUtensorMaps: FP32 A, then FP32 B
    int64_t nunits;
    int* err;
    long long timeout;
};
// Encodes the two FP32 tensor maps the fused split reads for one problem
// (A: K-contiguous rows lda floats apart, B: N-contiguous rows) into
// out[0..255]. lda and N multiples of 4, A and B 16-byte aligned.
bool tc_fused_maps(const float* A, int64_t lda, const float* B, int64_t M, int64_t K, int64_t N, void* out);
// Chunk length (k's per TMEM accumulation) the kernels use for K and a K split.
int tc_chunk_len(int64_t K, int splits);
cudaError_t tc_grouped_launch(const TcGroupArgs& g, int precision, int grid, cudaStream_t s);
// Bytes of the partial tiles / counters of one split problem of a grouped launch.
inline size_t tc_group_partial_floats(int64_t tiles, int splits) { return (size_t)tiles * splits * 128 * 128; }
constexpr int kTcGroupCountersPerTile = 8;

// Operand plane geometry. A planes are [P][M][Kp] (K-major). B planes are
// K-major [P][N][Kp] for TF32, N-major 128-byte panels [P][Np/NBE][K][NBE]
// for BF16. Kp pads K-major rows to 16 bytes, Np pads N to whole panels;
// padding holds zeros.
struct PlaneGeom {
    int P;                 // planes per operand: 2 (TF32) or 3 (BF16)
    int esize;             // bytes per plane element: 4 (TF32) or 2 (BF16)
    bool b_kmajor;         // B planes K-major (TF32) or N-major panels (BF16)
    int64_t Kp, Np;
    size_t a_plane_bytes, b_plane_bytes;   // one plane, rounded to 1 KiB
};
PlaneGeom plane_geom(int64_t M, int64_t K, int64_t N, int precision);
cudaError_t split_launch(const float* A, const float* B, int64_t M, int64_t K, int64_t N,
                         int precision, void* planes, cudaStream_t s);
// One matrix, laid out as the A operand (as_b false) or the B operand.
size_t split_one_bytes(int64_t R, int64_t C, int precision, bool as_b);
cudaError_t split_one(const float* X, int64_t R, int64_t C, int precision, bool as_b, void* out,
                      cudaStream_t s);

// Test probe: a wait that nothing ends, bounded by `limit` SM clocks.
cudaError_t tc_timeout_probe(int* err, long long limit, cudaStream_t s);

// Number of SMs of the current device (cached).
int device_sm_count();
// Device error word of the current device (allocated on first use).
int* device_error_word();

}  // namespace mmsk
