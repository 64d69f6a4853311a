// FP64 checking on the GPU: the product C64 = A*B in double from the FP32
// inputs, its absolute-value companion (|A||B|), and the error measures of an
// FP32 result against them.
//
// Not on the product path: no entry point that computes C = A*B calls these.
// They are the GPU form of the reference's FP64 checks, which compare every
// library against an FP64 product before timing (docs/BENCHMARKS.md:112-120,
// sampled FP64 dot products at :395-399), and of its checker
// Utils::check_correctness (common/utils.hpp:24-48). Large products (4096^3,
// the narrow-M shapes with K = 32768, the grouped batch) need an FP64 truth
// that a CPU loop cannot produce in the seconds a test may take.
//
// Arithmetic. Every C64[i][j] is one chain over k in increasing order,
// acc = fma((double)a_ik, (double)b_kj, acc) from +0. The product of two floats
// is exact in double (24 + 24 significant bits < 53), so each step rounds
// once, exactly as `acc += (double)a * (double)b` does on the CPU: C64 equals a
// sequential CPU loop over k bit for bit, whatever the tiling. (|A||B|)_ij is
// the same chain over |a_ik| |b_kj|.
//
// Error measures (one deterministic two-pass reduction: a fixed grid of
// blocks, each summing a fixed subset in a fixed order, then one block adding
// the block results in block order):
//   normwise = ||C - C64||_F / (||A||_F ||B||_F)
//   max_rel  = max |C - C64| / max(|C64|, 2^-24 (|A||B|)_ij)
//   rel_frob = ||C - C64||_F / ||C64||_F,   max_abs = max |C - C64|
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>

#include "internal.hpp"
#include "runtime.hpp"

namespace mmsk {
namespace {

constexpr int kDT = 64;          // output tile (64 x 64)
constexpr int kDK = 16;          // k per shared-memory stage
constexpr int kDThreads = 256;   // 16 x 16 threads, 4 x 4 outputs each

// C64 (and Cabs when ABS) for one 64 x 64 tile. Thread (ty, tx) owns rows
// ty + 16 i and columns tx + 16 j, so a warp reads two A values (broadcast)
// and sixteen consecutive B values per k. Loads outside the matrix read 0;
// steps past K are skipped, so every chain has exactly K terms.
template <bool ABS>
__global__ void __launch_bounds__(kDThreads)
dgemm_check_kernel(const float* __restrict__ A, const float* __restrict__ B, double* __restrict__ C,
                   double* __restrict__ Cabs, int64_t M, int64_t K, int64_t N) {
    __shared__ double As[kDK][kDT + 1];
    __shared__ double Bs[kDK][kDT];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t m0 = (int64_t)blockIdx.y * kDT, n0 = (int64_t)blockIdx.x * kDT;
    double acc[4][4], aab[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) { acc[i][j] = 0.0; aab[i][j] = 0.0; }

    for (int64_t k0 = 0; k0 < K; k0 += kDK) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int f = tid + r * kDThreads;          // 1024 = 64 rows x 16 k
            const int row = f / kDK, kk = f % kDK;
            const int64_t gm = m0 + row, gk = k0 + kk;
            As[kk][row] = (gm < M && gk < K) ? (double)A[gm * K + gk] : 0.0;
        }
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int f = tid + r * kDThreads;          // 1024 = 16 k x 64 columns
            const int kk = f / kDT, col = f % kDT;
            const int64_t gk = k0 + kk, gn = n0 + col;
            Bs[kk][col] = (gk < K && gn < N) ? (double)B[gk * N + gn] : 0.0;
        }
        __syncthreads();
        const int kmax = (int)((K - k0) < kDK ? (K - k0) : kDK);
#pragma unroll
        for (int kk = 0; kk < kDK; kk++) {
            if (kk < kmax) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
                for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        acc[i][j] = fma(a[i], b[j], acc[i][j]);
                        if constexpr (ABS) aab[i][j] = fma(fabs(a[i]), fabs(b[j]), aab[i][j]);
                    }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int64_t r = m0 + ty + 16 * i;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t c = n0 + tx + 16 * j;
            if (c >= N) continue;
            C[r * N + c] = acc[i][j];
            if constexpr (ABS) Cabs[r * N + c] = aab[i][j];
        }
    }
}

// Reduction layout: kErrBlocks blocks of kDThreads threads; block b, thread t
// visits elements b * kDThreads + t + s * kErrBlocks * kDThreads, s = 0, 1, ...
constexpr int kErrBlocks = 512;
constexpr int kErrSlots = 4;     // doubles per block result

// Sums in shared memory by halving, a fixed order for a fixed block size.
__device__ __forceinline__ void block_reduce(double* sh, int slots, bool is_max_slot[kErrSlots]) {
    for (int w = kDThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int s = 0; s < slots; s++) {
                const double x = sh[s * kDThreads + threadIdx.x], y = sh[s * kDThreads + threadIdx.x + w];
                sh[s * kDThreads + threadIdx.x] = is_max_slot[s] ? fmax(x, y) : x + y;
            }
        __syncthreads();
    }
}

// Per block: sum (C - C64)^2, sum C64^2, max |C - C64|, max relative error.
__global__ void __launch_bounds__(kDThreads)
err_partial_kernel(const float* __restrict__ Cf, const double* __restrict__ C64, const double* __restrict__ Cabs,
                   int64_t n, double* __restrict__ parts) {
    __shared__ double sh[kErrSlots * kDThreads];
    const double eps = 1.0 / 16777216.0;
    double sd = 0.0, sr = 0.0, ma = 0.0, mr = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kDThreads + threadIdx.x; i < n; i += (int64_t)kErrBlocks * kDThreads) {
        const double t = C64[i];
        const double e = fabs((double)Cf[i] - t);
        sd += e * e;
        sr += t * t;
        ma = fmax(ma, e);
        if (e > 0.0) {
            const double d = fabs(t);
            const double fl = Cabs ? eps * Cabs[i] : 0.0;
            const double den = d > fl ? d : fl;
            mr = fmax(mr, den > 0.0 ? e / den : (double)INFINITY);
        }
    }
    sh[0 * kDThreads + threadIdx.x] = sd;
    sh[1 * kDThreads + threadIdx.x] = sr;
    sh[2 * kDThreads + threadIdx.x] = ma;
    sh[3 * kDThreads + threadIdx.x] = mr;
    __syncthreads();
    bool is_max[kErrSlots] = {false, false, true, true};
    block_reduce(sh, kErrSlots, is_max);
    if (threadIdx.x == 0)
        for (int s = 0; s < kErrSlots; s++) parts[(size_t)blockIdx.x * kErrSlots + s] = sh[s * kDThreads];
}

// Per block: sum x^2 of an FP32 matrix (slot 0; the other slots 0).
__global__ void __launch_bounds__(kDThreads)
sumsq_partial_kernel(const float* __restrict__ X, int64_t n, double* __restrict__ parts) {
    __shared__ double sh[kErrSlots * kDThreads];
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kDThreads + threadIdx.x; i < n; i += (int64_t)kErrBlocks * kDThreads) {
        const double x = (double)X[i];
        s += x * x;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    bool is_max[kErrSlots] = {false, false, false, false};
    block_reduce(sh, 1, is_max);
    if (threadIdx.x == 0) {
        parts[(size_t)blockIdx.x * kErrSlots + 0] = sh[0];
        for (int k = 1; k < kErrSlots; k++) parts[(size_t)blockIdx.x * kErrSlots + k] = 0.0;
    }
}

// One block: the kErrBlocks block results of three reductions (C, A, B)
// combined in block order; out[0..5] = sum diff^2, sum C64^2, max abs,
// max rel, sum A^2, sum B^2.
__global__ void __launch_bounds__(kDThreads)
err_final_kernel(const double* __restrict__ parts, double* __restrict__ out) {
    __shared__ double sh[kErrSlots * kDThreads];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < kErrBlocks; b += kDThreads) {
        const double* pc = parts + (size_t)b * kErrSlots;
        const double* pa = parts + (size_t)(kErrBlocks + b) * kErrSlots;
        const double* pb = parts + (size_t)(2 * kErrBlocks + b) * kErrSlots;
        acc[0] += pc[0]; acc[1] += pc[1];
        acc[2] = fmax(acc[2], pc[2]); acc[3] = fmax(acc[3], pc[3]);
        acc[4] += pa[0]; acc[5] += pb[0];
    }
    // Two rounds of the four-slot block reduction: (0, 1, 2, 3), then (4, 5).
    for (int s = 0; s < 4; s++) sh[s * kDThreads + threadIdx.x] = acc[s];
    __syncthreads();
    bool is_max1[kErrSlots] = {false, false, true, true};
    block_reduce(sh, 4, is_max1);
    if (threadIdx.x == 0)
        for (int s = 0; s < 4; s++) out[s] = sh[s * kDThreads];
    __syncthreads();
    sh[threadIdx.x] = acc[4];
    sh[kDThreads + threadIdx.x] = acc[5];
    __syncthreads();
    bool is_max2[kErrSlots] = {false, false, false, false};
    block_reduce(sh, 2, is_max2);
    if (threadIdx.x == 0) { out[4] = sh[0]; out[5] = sh[kDThreads]; }
}

}  // namespace

size_t check_errors_work_bytes() { return (size_t)(3 * kErrBlocks * kErrSlots + 8) * sizeof(double); }

}  // namespace mmsk

using namespace mmsk;

extern "C" {

maxmulsk_status maxmulsk_check_dgemm_dev(const float* dA, const float* dB, double* dC64, double* dCabs, size_t M,
                                         size_t K, size_t N, void* stream) {
    if (M == 0 || N == 0) return MAXMULSK_OK;
    if (!dC64) { set_error_message("null C64"); return MAXMULSK_ERR_INVALID; }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (K == 0) {
        maxmulsk_status st = cuda_status(cudaMemsetAsync(dC64, 0, M * N * sizeof(double), s), "memset C64");
        if (st == MAXMULSK_OK && dCabs)
            st = cuda_status(cudaMemsetAsync(dCabs, 0, M * N * sizeof(double), s), "memset Cabs");
        return st;
    }
    if (!dA || !dB) { set_error_message("null matrix pointer"); return MAXMULSK_ERR_INVALID; }
    const size_t gy = (M + kDT - 1) / kDT, gx = (N + kDT - 1) / kDT;
    if (gy > 65535 || gx > 0x7FFFFFFFu || K > (size_t)INT64_MAX / 2) {
        set_error_message("shape too large for the FP64 check grid");
        return MAXMULSK_ERR_UNSUPPORTED;
    }
    const dim3 grid((unsigned)gx, (unsigned)gy);
    if (dCabs)
        dgemm_check_kernel<true><<<grid, kDThreads, 0, s>>>(dA, dB, dC64, dCabs, (int64_t)M, (int64_t)K, (int64_t)N);
    else
        dgemm_check_kernel<false><<<grid, kDThreads, 0, s>>>(dA, dB, dC64, nullptr, (int64_t)M, (int64_t)K,
                                                              (int64_t)N);
    return cuda_status(cudaGetLastError(), "FP64 check product launch");
}

size_t maxmulsk_check_errors_work_bytes(void) { return check_errors_work_bytes(); }

maxmulsk_status maxmulsk_check_errors_dev(const float* dC, const double* dC64, const double* dCabs,
                                          const float* dA, const float* dB, size_t M, size_t K, size_t N,
                                          void* work, size_t work_bytes, maxmulsk_error_report* out,
                                          void* stream) {
    if (!out) { set_error_message("null report"); return MAXMULSK_ERR_INVALID; }
    *out = maxmulsk_error_report{};
    if (M == 0 || N == 0) return MAXMULSK_OK;
    if (!dC || !dC64 || (K > 0 && (!dA || !dB))) { set_error_message("null pointer"); return MAXMULSK_ERR_INVALID; }
    if (!work || work_bytes < check_errors_work_bytes() || (reinterpret_cast<uintptr_t>(work) & 7) != 0) {
        set_error_message("work buffer missing, too small or not 8-byte aligned");
        return MAXMULSK_ERR_INVALID;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* parts = static_cast<double*>(work);
    double* res = parts + (size_t)3 * kErrBlocks * kErrSlots;
    err_partial_kernel<<<kErrBlocks, kDThreads, 0, s>>>(dC, dC64, dCabs, (int64_t)(M * N), parts);
    if (K > 0) {
        sumsq_partial_kernel<<<kErrBlocks, kDThreads, 0, s>>>(dA, (int64_t)(M * K), parts + (size_t)kErrBlocks * kErrSlots);
        sumsq_partial_kernel<<<kErrBlocks, kDThreads, 0, s>>>(dB, (int64_t)(K * N),
                                                              parts + (size_t)2 * kErrBlocks * kErrSlots);
    } else {
        maxmulsk_status st = cuda_status(
            cudaMemsetAsync(parts + (size_t)kErrBlocks * kErrSlots, 0, (size_t)2 * kErrBlocks * kErrSlots * sizeof(double), s),
            "memset partials");
        if (st != MAXMULSK_OK) return st;
    }
    err_final_kernel<<<1, kDThreads, 0, s>>>(parts, res);
    maxmulsk_status st = cuda_status(cudaGetLastError(), "FP64 error reduction launch");
    if (st != MAXMULSK_OK) return st;
    double h[6];
    st = cuda_status(cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, s), "read error report");
    if (st == MAXMULSK_OK) st = cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (st != MAXMULSK_OK) return st;
    out->norm_diff = std::sqrt(h[0]);
    out->norm_c64 = std::sqrt(h[1]);
    out->max_abs = h[2];
    out->max_rel = h[3];
    out->norm_a = std::sqrt(h[4]);
    out->norm_b = std::sqrt(h[5]);
    out->normwise = (h[4] > 0 && h[5] > 0) ? out->norm_diff / (out->norm_a * out->norm_b) : 0.0;
    out->rel_frob = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
    return MAXMULSK_OK;
}

}  // extern "C"
