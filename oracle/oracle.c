/*
 * CPU oracle for the row-major FP32 GEMM C = A*B.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product library links, loads or
 * calls this file; only the tests, the smoke check and the CPU-baseline leg of
 * the benchmark do. It is the checker, never the thing measured or shipped.
 *
 * Parity pin: oracle_sgemm_scalar restates Utils::multiply_scalar
 * (common/utils.hpp:50-61) and must agree with it bit for bit; the tests check
 * that against the reference's own header compiled here (oracle/_ref). The
 * reference ships no golden vectors, so the committed fixtures under
 * tests/golden/ were produced by running that compiled reference function on
 * seeded inputs (tests/golden/make_golden.py).
 *
 * Build: oracle/Makefile (gcc, -O2 -ffp-contract=off, no -march flags, so no
 * FMA is contracted and every float operation is the IEEE one written here).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Counter-based inputs. The same formulas run in numpy (maxmulsk_b200.datagen) */
/* so host and device see identical bytes. SplitMix64 of (seed, index).        */
/* ------------------------------------------------------------------------- */
static inline uint64_t splitmix64(uint64_t seed, uint64_t idx) {
    uint64_t z = seed + (idx + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* U[-1,1): the top 24 bits as an integer u, x = (u - 2^23) * 2^-23 (exact). */
void oracle_fill_uniform(float* x, size_t n, uint64_t seed) {
    for (size_t i = 0; i < n; i++) {
        int32_t u = (int32_t)(splitmix64(seed, i) >> 40);
        x[i] = (float)(u - 8388608) * (1.0f / 8388608.0f);
    }
}

/* Approximately N(0, scale^2): Irwin-Hall sum of 12 24-bit uniforms, summed in
 * integers (exact), centred, converted once (round to nearest), scaled. */
void oracle_fill_normal(float* x, size_t n, uint64_t seed, float scale) {
    for (size_t i = 0; i < n; i++) {
        int64_t s = 0;
        for (int j = 0; j < 12; j++) s += (int64_t)(splitmix64(seed, i * 12ull + (uint64_t)j) >> 40);
        s -= 6ll * 16777216ll;
        float z = (float)s * (1.0f / 16777216.0f);
        x[i] = z * scale;
    }
}

/* Wide-range: uniform 23-bit mantissa, exponent uniform in [-20, 20], random
 * sign, assembled from bits (no libm). */
void oracle_fill_wide(float* x, size_t n, uint64_t seed) {
    for (size_t i = 0; i < n; i++) {
        uint64_t z = splitmix64(seed, i);
        uint32_t sign = (uint32_t)(z >> 63) << 31;
        int32_t e = (int32_t)(((z >> 32) & 0xFFFFull) % 41ull) - 20;
        uint32_t mant = (uint32_t)(z & 0x7FFFFFull);
        uint32_t bits = sign | ((uint32_t)(127 + e) << 23) | mant;
        memcpy(&x[i], &bits, 4);
    }
}

/* ------------------------------------------------------------------------- */
/* FP32 products                                                              */
/* ------------------------------------------------------------------------- */

/* Restates Utils::multiply_scalar (common/utils.hpp:50-61): i, j, k loop
 * order, one float accumulator per output, separate multiply and add (no FMA),
 * k summed in increasing order. NOTE the argument order (M, N, K) of the
 * original. */
void oracle_sgemm_scalar(const float* A, const float* B, float* C,
                         size_t M, size_t N, size_t K) {
    for (size_t i = 0; i < M; ++i) {
        for (size_t j = 0; j < N; ++j) {
            float sum = 0.0f;
            for (size_t k = 0; k < K; ++k) {
                float p = A[i * K + k] * B[k * N + j];
                sum = sum + p;
            }
            C[i * N + j] = sum;
        }
    }
}

/* The outer-Kc panel order of the reference's v3 driver
 * (sme/v3/sme-1x4-acc-kcout.cpp:464-471 first_k, :530-558 store/store_add):
 * each Kc panel p_t is an independent sum over its k range; the first panel
 * overwrites C, each later one is added into what is there, so
 * C = ((p0 + p1) + p2) + ...
 * Within a panel the sum runs k upward. With fma != 0 each step is one fused
 * multiply-add (fmaf), which is how the CUDA SIMT kernel accumulates; with
 * fma == 0 it is a multiply then an add, as in multiply_scalar. Arguments in
 * the C ABI's (M, K, N) order. kc == 0 means one panel (kc = K). */
void oracle_sgemm_panels(const float* A, const float* B, float* C,
                         size_t M, size_t K, size_t N, size_t kc, int fma) {
    if (kc == 0 || kc > K) kc = K;
    for (size_t i = 0; i < M; ++i) {
        for (size_t j = 0; j < N; ++j) {
            float c = 0.0f;
            for (size_t kk = 0; kk < K; kk += kc) {
                size_t ke = kk + kc < K ? kk + kc : K;
                float p = 0.0f;
                if (fma) {
                    for (size_t k = kk; k < ke; ++k) p = fmaf(A[i * K + k], B[k * N + j], p);
                } else {
                    for (size_t k = kk; k < ke; ++k) { float t = A[i * K + k] * B[k * N + j]; p = p + t; }
                }
                c = (kk == 0) ? p : c + p;
            }
            C[i * N + j] = c;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* FP64 truth: C64 = A*B from the same FP32 inputs, (M, K, N) order.           */
/* Row blocks on pthreads; each row is computed by one thread in i, k, j order  */
/* so the result does not depend on the thread count.                         */
/* ------------------------------------------------------------------------- */
typedef struct {
    const float* A; const float* B; double* C;
    size_t K, N, r0, r1;
} dgemm_job;

/* One FP64 row: dst[j] = sum_k A[i][k] * B[k][j], k upward. */
static void dgemm_one_row(const float* A, const float* B, double* dst,
                          size_t K, size_t N, size_t i) {
    for (size_t c = 0; c < N; c++) dst[c] = 0.0;
    for (size_t k = 0; k < K; k++) {
        double a = (double)A[i * K + k];
        const float* b = B + k * N;
        for (size_t c = 0; c < N; c++) dst[c] += a * (double)b[c];
    }
}

static void* dgemm_rows(void* p) {
    dgemm_job* j = (dgemm_job*)p;
    for (size_t i = j->r0; i < j->r1; i++) dgemm_one_row(j->A, j->B, j->C + i * j->N, j->K, j->N, i);
    return NULL;
}

void oracle_dgemm(const float* A, const float* B, double* C,
                  size_t M, size_t K, size_t N, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if ((size_t)nthreads > M) nthreads = (int)(M ? M : 1);
    pthread_t th[256];
    dgemm_job jobs[256];
    if (nthreads > 256) nthreads = 256;
    size_t per = (M + (size_t)nthreads - 1) / (size_t)nthreads;
    int launched = 0;
    for (int t = 0; t < nthreads; t++) {
        size_t r0 = (size_t)t * per, r1 = r0 + per < M ? r0 + per : M;
        if (r0 >= r1) break;
        jobs[t] = (dgemm_job){A, B, C, K, N, r0, r1};
        if (nthreads == 1) { dgemm_rows(&jobs[t]); continue; }
        pthread_create(&th[t], NULL, dgemm_rows, &jobs[t]);
        launched++;
    }
    for (int t = 0; t < launched; t++) pthread_join(th[t], NULL);
}

/* (|A||B|)_ij in FP64, one row after another, k upward: the floor of the
 * max-relative measure below, formed for every element (the GPU check
 * product's companion output is compared with it bit for bit). */
void oracle_dgemm_abs(const float* A, const float* B, double* C, size_t M, size_t K, size_t N) {
    for (size_t i = 0; i < M; i++) {
        double* dst = C + i * N;
        for (size_t c = 0; c < N; c++) dst[c] = 0.0;
        for (size_t k = 0; k < K; k++) {
            double a = fabs((double)A[i * K + k]);
            const float* b = B + k * N;
            for (size_t c = 0; c < N; c++) dst[c] += a * fabs((double)b[c]);
        }
    }
}

/* FP64 value of selected rows only (sampled checks of large products). */
void oracle_dgemm_rows(const float* A, const float* B, double* C,
                       size_t K, size_t N, const int64_t* rows, size_t nrows) {
    for (size_t r = 0; r < nrows; r++) dgemm_one_row(A, B, C + r * N, K, N, (size_t)rows[r]);
}

/* ------------------------------------------------------------------------- */
/* Error measures                                                             */
/* ------------------------------------------------------------------------- */

/* out[0] normwise   = ||C - C64||_F / (||A||_F * ||B||_F)
 * out[1] max elementwise relative = max |C - C64| / max(|C64|, eps * (|A||B|)_ij)
 *        with eps = 2^-24; (|A||B|)_ij is only formed when |C64| is below it, so
 *        the cost stays O(MN) plus O(K) per such element.
 * out[2] relative Frobenius = ||C - C64||_F / ||C64||_F
 * out[3] max |C - C64|                                                        */
void oracle_errors(const float* C, const double* C64, const float* A, const float* B,
                   size_t M, size_t K, size_t N, double* out) {
    double num = 0, den = 0, na = 0, nb = 0, maxrel = 0, maxabs = 0;
    const double eps = 1.0 / 16777216.0;
    for (size_t i = 0; i < M * K; i++) na += (double)A[i] * A[i];
    for (size_t i = 0; i < K * N; i++) nb += (double)B[i] * B[i];
    for (size_t i = 0; i < M; i++) {
        for (size_t j = 0; j < N; j++) {
            double t = C64[i * N + j];
            double e = fabs((double)C[i * N + j] - t);
            num += e * e;
            den += t * t;
            if (e > maxabs) maxabs = e;
            double d = fabs(t);
            if (e > 0) {
                /* only when it can matter: floor = eps * sum_k |a_ik||b_kj| */
                if (e / (d > 0 ? d : 1e-300) > maxrel) {
                    double s = 0;
                    for (size_t k = 0; k < K; k++) s += fabs((double)A[i * K + k]) * fabs((double)B[k * N + j]);
                    double fl = eps * s;
                    double q = e / (d > fl ? d : fl);
                    if (q > maxrel) maxrel = q;
                }
            }
        }
    }
    out[0] = (na > 0 && nb > 0) ? sqrt(num) / (sqrt(na) * sqrt(nb)) : 0.0;
    out[1] = maxrel;
    out[2] = den > 0 ? sqrt(num / den) : 0.0;
    out[3] = maxabs;
}

/* Relative Frobenius distance between two FP32 results, the measure of the
 * reference's v4-vs-v3 checker (bench/results/2026-09-13/source/check_nb.cpp:14-18). */
double oracle_relfrob(const float* a, const float* b, size_t n) {
    double num = 0, den = 0;
    for (size_t i = 0; i < n; i++) {
        double e = (double)a[i] - (double)b[i];
        num += e * e;
        den += (double)b[i] * b[i];
    }
    return den > 0 ? sqrt(num / den) : 0.0;
}

/* Restates Utils::check_correctness (common/utils.hpp:24-48) without the
 * printing: number of entries with |ref - got| > tol, and the largest such
 * difference in *max_diff. */
size_t oracle_check_correctness(const float* ref, const float* got, size_t n, float tol,
                                float* max_diff) {
    size_t bad = 0;
    float md = 0.0f;
    for (size_t i = 0; i < n; i++) {
        float d = fabsf(ref[i] - got[i]);
        if (d > tol) { bad++; if (d > md) md = d; }
    }
    if (max_diff) *max_diff = md;
    return bad;
}

/* ------------------------------------------------------------------------- */
/* Split-precision operand planes, from their definitions                     */
/* ------------------------------------------------------------------------- */

/* TF32 round-to-nearest, ties away from zero, kept as an FP32 bit pattern
 * with the low 13 mantissa bits clear: add half an ulp of the 10-bit mantissa
 * to the magnitude bits, then truncate. Finite inputs only. */
static inline float tf32_rna(float x) {
    uint32_t b; memcpy(&b, &x, 4);
    b = (b + 0x1000u) & 0xFFFFE000u;
    float r; memcpy(&r, &b, 4);
    return r;
}

/* BF16 round-to-nearest-even, returned widened to FP32. Finite inputs only. */
static inline float bf16_rne(float x) {
    uint32_t b; memcpy(&b, &x, 4);
    b = (b + 0x7FFFu + ((b >> 16) & 1u)) & 0xFFFF0000u;
    float r; memcpy(&r, &b, 4);
    return r;
}

/* x = hi + lo + O(2^-22 |x|): hi = tf32(x), lo = tf32(x - hi). */
void oracle_split_tf32(const float* x, float* hi, float* lo, size_t n) {
    for (size_t i = 0; i < n; i++) {
        float h = tf32_rna(x[i]);
        hi[i] = h;
        lo[i] = tf32_rna(x[i] - h);
    }
}

/* x = l0 + l1 + l2 (+ a remainder of at most 2^-24 |x|): each limb is the
 * BF16 rounding of what the previous limbs left. Limbs returned as FP32. */
void oracle_split_bf16(const float* x, float* l0, float* l1, float* l2, size_t n) {
    for (size_t i = 0; i < n; i++) {
        float a = bf16_rne(x[i]);
        float r1 = x[i] - a;
        float b = bf16_rne(r1);
        float r2 = r1 - b;
        l0[i] = a; l1[i] = b; l2[i] = bf16_rne(r2);
    }
}

/* The split product without any accumulation error: C = sum over the kept
 * limb pairs, accumulated in FP64, then rounded once to FP32.
 * mode 1: 3xTF32 (hi*hi + hi*lo + lo*hi); mode 2: BF16x6 (limb pairs with
 * i + j <= 2); mode 3: BF16x9 (all nine pairs). (M, K, N) order. */
void oracle_sgemm_split_exact(const float* A, const float* B, float* C,
                              size_t M, size_t K, size_t N, int mode) {
    size_t na = M * K, nb = K * N;
    float* a[3]; float* b[3];
    for (int p = 0; p < 3; p++) { a[p] = (float*)calloc(na ? na : 1, 4); b[p] = (float*)calloc(nb ? nb : 1, 4); }
    int planes;
    if (mode == 1) {
        oracle_split_tf32(A, a[0], a[1], na);
        oracle_split_tf32(B, b[0], b[1], nb);
        planes = 2;
    } else {
        oracle_split_bf16(A, a[0], a[1], a[2], na);
        oracle_split_bf16(B, b[0], b[1], b[2], nb);
        planes = 3;
    }
    double* acc = (double*)malloc((N ? N : 1) * sizeof(double));
    for (size_t i = 0; i < M; i++) {
        for (size_t j = 0; j < N; j++) acc[j] = 0.0;
        for (int pa = 0; pa < planes; pa++) {
            for (int pb = 0; pb < planes; pb++) {
                int keep = (mode == 1) ? (pa + pb <= 1) : (mode == 2) ? (pa + pb <= 2) : 1;
                if (!keep) continue;
                for (size_t k = 0; k < K; k++) {
                    double av = (double)a[pa][i * K + k];
                    const float* br = b[pb] + k * N;
                    for (size_t j = 0; j < N; j++) acc[j] += av * (double)br[j];
                }
            }
        }
        for (size_t j = 0; j < N; j++) C[i * N + j] = (float)acc[j];
    }
    free(acc);
    for (int p = 0; p < 3; p++) { free(a[p]); free(b[p]); }
}
