#pragma once
/*
 * MaxMulSK-B200: row-major FP32 GEMM C = A*B on NVIDIA B200 (sm_100a).
 *
 * Drop-in for the reference's C ABI (capi/maxmulsk.h:9-41). Every function
 * computes C = A*B for row-major, tightly packed FP32 matrices: A is M x K,
 * B is K x N, C is M x N. C is overwritten (alpha = 1, beta = 0); its previous
 * contents are never read. Dimensions follow the reference's (M, K, N) order,
 * not BLAS's (M, N, K).
 *
 * Empty shapes follow the reference (capi/maxmulsk.cpp:13-20): M == 0 or
 * N == 0 returns MAXMULSK_OK without touching anything; K == 0 sets C to zero.
 *
 * The header names no CUDA type. A stream is passed as `void*` holding a
 * cudaStream_t (NULL = the legacy default stream). Device pointers are plain
 * pointers to memory of the current CUDA device.
 *
 * Thread safety: calls from several host threads are safe. Workspace is kept
 * per (device, stream); the tuning database is loaded once under a mutex.
 */
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The first three keep the reference's values
 * (capi/maxmulsk.h:24-28); the rest are appended, never renumbered. */
typedef enum {
    MAXMULSK_OK = 0,
    MAXMULSK_ERR_UNSUPPORTED,   /* the plan or shape was rejected; C untouched   */
    MAXMULSK_ERR_ALLOC,         /* a device or pinned buffer could not be had     */
    MAXMULSK_ERR_CUDA,          /* a CUDA runtime/driver call failed              */
    MAXMULSK_ERR_INVALID,       /* a null pointer, or a workspace that is too small */
    MAXMULSK_ERR_TIMEOUT,       /* a bounded device-side wait gave up             */
} maxmulsk_status;

/* ----------------------------------------------------------------------------
 * Drop-in entry points (host pointers, synchronous, FP32-SIMT accurate).
 * Each copies A and B to the current device, multiplies, copies C back and
 * waits. With page-locked A and C (cudaHostAlloc / cudaHostRegister) of at
 * least 1024 rows and 32 MiB, the copies run as a pipeline of row blocks that
 * overlaps them with the GEMM; pageable buffers are copied whole, through the
 * CUDA runtime's own staging.
 * ------------------------------------------------------------------------- */

/* Replaces capi/maxmulsk.h:32-33 (SMEKernels1x4AccKcOut). The plan comes from
 * the tuning picker, FP32 SIMT precision; MAXMULSK_CONFIG overrides it. The
 * picker: the tuning database; else, when the learned cost model cannot be
 * trusted for the shape (see maxmulsk_picker_doubt), an exhaustive search of
 * the candidates on the call's own operands (device copies of them for host
 * pointers; never inside a stream capture) whose winner enters the database;
 * else the learned model; else the shape rule. Unlike the reference's v3,
 * allocation failure is reported (MAXMULSK_ERR_ALLOC). */
maxmulsk_status maxmulsk_sgemm_v3(const float* A, const float* B, float* C,
                                  size_t M, size_t K, size_t N);

/* Replaces capi/maxmulsk.h:36-37 (the v4c dispatcher): a fixed shape rule
 * picks between two plans, as sme/v4/sme-1x4-v4c-dispatch.cpp:17-22 does;
 * no database and no environment override. FP32 SIMT precision. */
maxmulsk_status maxmulsk_sgemm_v4(const float* A, const float* B, float* C,
                                  size_t M, size_t K, size_t N);

/* ----------------------------------------------------------------------------
 * Device-pointer variants: asynchronous on `stream`. Errors detected on the
 * host are returned at once; a device-side timeout is reported by
 * maxmulsk_stream_status().
 * ------------------------------------------------------------------------- */
maxmulsk_status maxmulsk_sgemm_v3_dev(const float* dA, const float* dB, float* dC,
                                      size_t M, size_t K, size_t N, void* stream);
maxmulsk_status maxmulsk_sgemm_v4_dev(const float* dA, const float* dB, float* dC,
                                      size_t M, size_t K, size_t N, void* stream);

/* ----------------------------------------------------------------------------
 * Precision and plans.
 * ------------------------------------------------------------------------- */
typedef enum {
    MAXMULSK_PREC_FP32   = 0,   /* FP32 FMA on the CUDA cores                    */
    MAXMULSK_PREC_3XTF32 = 1,   /* tensor cores: hi*hi + hi*lo + lo*hi, TF32      */
    MAXMULSK_PREC_BF16X6 = 2,   /* tensor cores: 3 BF16 limbs, pairs i+j <= 2     */
    MAXMULSK_PREC_BF16X9 = 3,   /* tensor cores: 3 BF16 limbs, all nine pairs     */
    MAXMULSK_PREC_SPLIT_AUTO = 4, /* tensor cores, the picker chooses 3XTF32 or
                                     BF16X6 (both within 2x the FP32 kernel's error) */
} maxmulsk_precision;

/* Kernel variants inside MAXMULSK_PREC_FP32. */
enum {
    MAXMULSK_FP32_FMA    = 0,   /* one fused multiply-add per k step             */
    MAXMULSK_FP32_SCALAR = 1,   /* multiply then add per k step, the arithmetic of
                                   Utils::multiply_scalar (common/utils.hpp:50-61) */
};

/* Variants of the tensor-core precisions. */
enum {
    MAXMULSK_TC_SPLIT_INPUTS = 0,  /* split A and B into operand planes, then multiply */
    MAXMULSK_TC_REUSE_PLANES = 1,  /* the workspace already holds the planes of these
                                      A and B (a previous call with the same inputs,
                                      shape, precision and workspace): skip the split */
    MAXMULSK_TC_FUSED_SPLIT = 2,   /* split inside the GEMM kernel: FP32 tiles of A and
                                      B are loaded and cut into limbs on the fly, with
                                      no planes in memory. BF16X6 / BF16X9, 128 x 128
                                      tiles, K and N multiples of 4. Pointers that are
                                      not 16-byte aligned run the split-inputs path
                                      (same result), so the workspace is sized for it */
};

/* The analog of the reference's Blocking (sme/v4/sme-1x4-kcout-ncblock-apack4za.hpp:30,
 * sme/support/gemm_tuning.hpp:37-43): how one GEMM is cut into work.
 *   precision : maxmulsk_precision
 *   tile_m, tile_n : output tile. FP32 (one CTA): 128x128, 128x64, 64x64.
 *                    Tensor cores: 128 x {64, 128, 256} on one CTA, or
 *                    256 x {128, 256} on a pair of CTAs (tcgen05 cta_group::2).
 *   split_k   : number of K slices (1..64). Slices are summed in slice order,
 *               first slice first, like the reference's outer-Kc panels
 *               (sme/v3/sme-1x4-acc-kcout.cpp:464-471, 530-558). Tensor-core
 *               plans also take 0: as many slices per tile as the device has
 *               work slots (SMs, or CTA pairs) per tile, at most 64, so one
 *               launch runs about one equal K slice per SM.
 *   variant   : FP32: MAXMULSK_FP32_FMA or MAXMULSK_FP32_SCALAR.
 *               Tensor cores: MAXMULSK_TC_SPLIT_INPUTS, MAXMULSK_TC_REUSE_PLANES or
 *               MAXMULSK_TC_FUSED_SPLIT.
 *   chunk     : tensor cores only: k's accumulated in TMEM before the epilogue
 *               adds them into FP32 registers (round to nearest, in k order) --
 *               the counterpart of the reference's Kc panel, whose partial
 *               products are added into C panel after panel. A multiple of 32
 *               in 32 .. 4096; 0 = chosen by K (shorter chunks cost more
 *               drains and give less error). FP32 plans: 0.
 *   reserved  : zero. */
typedef struct {
    int32_t precision;
    int32_t tile_m;
    int32_t tile_n;
    int32_t split_k;
    int32_t variant;
    int32_t chunk;
    int32_t reserved[2];
} maxmulsk_plan;

/* Validates a plan for a shape (the analog of NB::classify,
 * sme/v4/sme-1x4-kcout-ncblock-apack4za.cpp:410-423): MAXMULSK_OK or
 * MAXMULSK_ERR_UNSUPPORTED. A rejected plan never touches C. */
maxmulsk_status maxmulsk_classify(size_t M, size_t K, size_t N, const maxmulsk_plan* plan);

/* The picker behind maxmulsk_sgemm_v3 for a given precision (the analog of
 * MaxMulSK::tuning::select, sme/support/gemm_tuning.cpp:96-100), as a query:
 * MAXMULSK_CONFIG, the tuning database, the learned model, the rule. It has
 * no operands, so it never searches; after a GEMM call on the shape ran the
 * exhaustive fallback, it returns that call's plan (now in the database). */
maxmulsk_status maxmulsk_choose(size_t M, size_t K, size_t N, int32_t precision,
                                maxmulsk_plan* out);

/* Why the GEMM entry points would run the exhaustive search for this shape
 * and precision instead of trusting the learned model: "no learned model",
 * "shape outside the trained range" (M, N or K above 16384), "close call"
 * (its two best candidates predicted within MAXMULSK_AUTOTUNE_MARGIN, default
 * 0.005 in ln-time). NULL when the tuning database or the model decides, for
 * BF16X9 (not searched), or with MAXMULSK_AUTOTUNE=0 (fallback off). The
 * counterpart in the reference is the MAXMULSK_BLOCKING sweep override
 * (sme/support/gemm_tuning.cpp:66-78). */
const char* maxmulsk_picker_doubt(size_t M, size_t K, size_t N, int32_t precision);

/* The fixed shape rule behind maxmulsk_sgemm_v4 (the analog of
 * SMEKernels1x4V4C::choose, sme/v4/sme-1x4-v4c-dispatch.cpp:17-22). */
maxmulsk_status maxmulsk_choose_rule(size_t M, size_t K, size_t N, int32_t precision,
                                     maxmulsk_plan* out);

/* Device workspace a plan needs (the analog of workspace_bytes,
 * sme/v5/sme-1x4-fusedpack-v51.hpp:75-78, and NB::capacity,
 * sme/v4/sme-1x4-kcout-ncblock-apack4za.cpp:429-444). 0 when none. */
size_t maxmulsk_workspace_bytes(size_t M, size_t K, size_t N, const maxmulsk_plan* plan);

/* Explicit plan, caller-owned device workspace (no allocation inside the
 * call; the analog of run_multiplication_ws, sme/v5/sme-1x4-fusedpack-v51.hpp:76-78).
 * ws must be 256-byte aligned and at least maxmulsk_workspace_bytes() long;
 * ws may be NULL when that is 0. Asynchronous on `stream`. */
maxmulsk_status maxmulsk_sgemm_plan_dev(const float* dA, const float* dB, float* dC,
                                        size_t M, size_t K, size_t N,
                                        const maxmulsk_plan* plan,
                                        void* ws, size_t ws_bytes, void* stream);

/* Explicit plan on host pointers, synchronous (workspace managed inside). */
maxmulsk_status maxmulsk_sgemm_plan(const float* A, const float* B, float* C,
                                    size_t M, size_t K, size_t N,
                                    const maxmulsk_plan* plan);

/* Split-precision tensor-core GEMM, selected explicitly (the plain names stay
 * FP32 SIMT). precision is one of MAXMULSK_PREC_3XTF32 / _BF16X6 / _BF16X9, or
 * MAXMULSK_PREC_SPLIT_AUTO to let the picker choose the split count. The
 * plan comes from the picker as for maxmulsk_sgemm_v3 (exhaustive fallback
 * included); MAXMULSK_CONFIG overrides it when its precision is the one asked. */
maxmulsk_status maxmulsk_sgemm_split(const float* A, const float* B, float* C,
                                     size_t M, size_t K, size_t N, int32_t precision);
maxmulsk_status maxmulsk_sgemm_split_dev(const float* dA, const float* dB, float* dC,
                                         size_t M, size_t K, size_t N, int32_t precision,
                                         void* stream);

/* TEST ONLY: writes the operand planes the split pre-pass makes from one
 * row-major R x C FP32 matrix, exactly as the tensor-core path does (the
 * analog of NB::probe_pack_A / probe_pack_B,
 * sme/v4/sme-1x4-kcout-ncblock-apack4za.hpp:44-49). Planes are FP32 (3xTF32,
 * P = 2) or BF16 (P = 3), each plane starting at a multiple of 1 KiB.
 *   as_b == 0 (A operand, R x C = M x K): [P][R][Cp], Cp = C padded to 16 bytes.
 *   as_b != 0 (B operand, R x C = K x N):
 *     3xTF32: transposed, K-major [P][C][Rp], Rp = R padded to 16 bytes;
 *     BF16:   N-major panels [P][Cp/NBE][R][NBE], NBE = 64, Cp = C padded to 64.
 * out must hold maxmulsk_probe_split_bytes() bytes. Asynchronous on `stream`. */
size_t maxmulsk_probe_split_bytes(size_t R, size_t C, int32_t precision, int32_t as_b);
maxmulsk_status maxmulsk_probe_split_dev(const float* dX, size_t R, size_t C, int32_t precision,
                                         int32_t as_b, void* out, void* stream);

/* TEST ONLY: launches one thread that waits, with the bounded wait every
 * kernel of this library uses, on a barrier that nothing completes, for
 * `cycles` SM clocks (1 .. 2e9); the timeout is then recorded in the device
 * error word, which the next maxmulsk_stream_status(stream) reports as
 * MAXMULSK_ERR_TIMEOUT and clears. No reference counterpart: the reference
 * runs on the CPU and has no device-side waits. */
maxmulsk_status maxmulsk_probe_timeout_dev(int64_t cycles, void* stream);

/* ----------------------------------------------------------------------------
 * Grouped launches: many independent GEMMs in one persistent kernel, captured
 * in a CUDA graph. The counterpart of run_batch(const Gemm*, size_t)
 * (sme/v3/sme-1x4-acc-kcout-onestream.hpp:61-63), same fields in the same
 * order; pointers are device pointers that must stay valid while the group
 * exists.
 * ------------------------------------------------------------------------- */
typedef struct {
    const float* A;
    const float* B;
    float* C;
    size_t M, K, N;
} maxmulsk_problem;

typedef struct maxmulsk_grouped_s* maxmulsk_grouped;

/* Plans the group, uploads its tables, allocates its scratch and captures one
 * CUDA graph. Call with the device current and the problems' buffers idle.
 * group_plan NULL, or an FP32 plan: the FP32 grouped kernel. Its tile (one per
 * group; NULL = chosen) and K split (split_k > 0 = that split for every
 * problem, 0 = chosen per problem) are what the caller gives; what is left
 * open is chosen by timing candidate configurations of the whole group (tile
 * shape x K-split policy), each captured and replayed, the fastest kept --
 * the group-level form of maxmulsk_autotune_dev. The search runs the group,
 * so C is written while the group is created.
 * A group_plan of precision MAXMULSK_PREC_BF16X6 / _BF16X9 / _SPLIT_AUTO runs
 * the problems on the fused-split tensor-core kernel, 128 x 128 tiles (tile
 * and variant fields are ignored). With split_k 0 the search also decides
 * which large problems run instead as their own launches of their picked plan
 * (split pre-pass + tcgen05 GEMM, 3xTF32 allowed under SPLIT_AUTO) inside
 * the same graph. An A with K not a multiple of 4 (or not 16-byte aligned) is
 * copied to a padded buffer of the group inside the graph; problems with N
 * not a multiple of 4, or B not 16-byte aligned, run in the FP32 SIMT part of
 * the same graph, at FP32 accuracy. maxmulsk_grouped_plans tells each
 * problem's plan. */
maxmulsk_status maxmulsk_grouped_create(const maxmulsk_problem* problems, size_t count,
                                        const maxmulsk_plan* group_plan, maxmulsk_grouped* out);
/* Replays the captured graph on `stream` (asynchronous). */
maxmulsk_status maxmulsk_grouped_launch(maxmulsk_grouped g, void* stream);
/* The plan chosen: group tile shape, per-problem split_k (count entries, may
 * be NULL), number of work units. */
maxmulsk_status maxmulsk_grouped_info(maxmulsk_grouped g, maxmulsk_plan* group_plan, int32_t* split_k,
                                      size_t* units);
/* The plan each problem runs (count entries): FP32 problems the group's tile,
 * their K split and variant; fused problems (precision, 128, 128, K split,
 * MAXMULSK_TC_FUSED_SPLIT) -- for an A repacked to a padded pitch the result
 * is that of MAXMULSK_TC_SPLIT_INPUTS on the same tiles; problems run as their
 * own launches, their plan. Each problem's C equals a single launch of its
 * plan bit for bit. */
maxmulsk_status maxmulsk_grouped_plans(maxmulsk_grouped g, maxmulsk_plan* plans);
void maxmulsk_grouped_destroy(maxmulsk_grouped g);
/* One-shot: create, launch on `stream`, wait, destroy. */
maxmulsk_status maxmulsk_sgemm_grouped_dev(const maxmulsk_problem* problems, size_t count, void* stream);

/* ----------------------------------------------------------------------------
 * Autotuner, tuning database and learned cost model.
 * The reference's picker is a static table plus an environment override
 * (sme/support/gemm_tuning.cpp:34-100) and a fixed rule
 * (sme/v4/sme-1x4-v4c-dispatch.cpp:17-22). Here: an exhaustive autotuner over
 * a fixed candidate list, a tuning database of its results, and a small MLP
 * trained on its timings that predicts every candidate's log-time.
 * Class 0 = FP32 candidates (24), class 1 = split-precision candidates (48).
 * ------------------------------------------------------------------------- */
#define MAXMULSK_MLP_FEATURES 7
#define MAXMULSK_MLP_HIDDEN 64
#define MAXMULSK_MLP_OUTPUTS 48
#define MAXMULSK_MLP_PARAMS (7 * 64 + 64 + 64 * 64 + 64 + 64 * 48 + 48)

/* The candidate plans of a class; returns how many were written (<= cap). */
size_t maxmulsk_candidates(int32_t cls, maxmulsk_plan* out, size_t cap);

/* Times each plan on one shape (device inputs, caller workspace): median of a
 * CUDA-graph replay of `reps` calls (reps <= 0: chosen per plan). Writes
 * microseconds per call to times_us; INFINITY for a plan the shape rejects or
 * whose workspace exceeds ws_bytes. Synchronises `stream`. */
maxmulsk_status maxmulsk_autotune_time_dev(const float* dA, const float* dB, float* dC,
                                           size_t M, size_t K, size_t N,
                                           const maxmulsk_plan* plans, size_t nplans,
                                           void* ws, size_t ws_bytes, int32_t reps,
                                           float* times_us, void* stream);

/* Exhaustive search over the candidates for `precision` (FP32, SPLIT_AUTO, or
 * one split mode); the best plan is returned and stored in the tuning
 * database under (M, K, N, precision). */
maxmulsk_status maxmulsk_autotune_dev(const float* dA, const float* dB, float* dC,
                                      size_t M, size_t K, size_t N, int32_t precision,
                                      void* ws, size_t ws_bytes, maxmulsk_plan* best,
                                      float* best_us, void* stream);

/* Tuning database (text; MAXMULSK_TUNING_DB is read on first use). */
int32_t maxmulsk_tuning_load(const char* path);   /* entries read, or -1 */
int32_t maxmulsk_tuning_save(const char* path);   /* entries written, or -1 */
void maxmulsk_tuning_clear(void);

/* Learned cost model: load weights (MAXMULSK_MODEL is read on first use);
 * NULL unloads. */
maxmulsk_status maxmulsk_model_load(const char* path);
/* The model's features of a shape, and its predicted log-times on the host. */
maxmulsk_status maxmulsk_mlp_features(size_t M, size_t K, size_t N, int32_t cls, float* out);
maxmulsk_status maxmulsk_mlp_predict_host(size_t M, size_t K, size_t N, int32_t cls, float* out);

/* Training and batched inference kernels (device pointers, float32, row-major).
 * params: MAXMULSK_MLP_PARAMS floats W1[F][H] b1 W2[H][H] b2 W3[H][O] b3.
 * forward: X[B][F] -> Z1, H1, Z2, H2 [B][H], Y[B][O] (Z1/Z2 may be NULL).
 * backward: masked MSE over the entries with mask != 0, divided by `count`;
 *   grads like params; work >= B * (O + 2H) floats; rowloss[B] squared errors.
 * adam: one bias-corrected Adam step (step >= 1) on params.
 * predict: Y[B][O]; with mask, best[B] = masked argmin (-1 if none);
 *   work >= 2 * B * H floats. */
maxmulsk_status maxmulsk_mlp_forward_dev(const float* params, const float* X, int32_t B, float* Z1, float* H1,
                                         float* Z2, float* H2, float* Y, void* stream);
maxmulsk_status maxmulsk_mlp_backward_dev(const float* params, const float* X, const float* Z1, const float* H1,
                                          const float* Z2, const float* H2, const float* Y, const float* T,
                                          const float* mask, int32_t B, float count, float* grads, float* work,
                                          float* rowloss, void* stream);
maxmulsk_status maxmulsk_mlp_adam_dev(float* params, const float* grads, float* m, float* v, float lr,
                                      float beta1, float beta2, float eps, int32_t step, void* stream);
maxmulsk_status maxmulsk_mlp_predict_dev(const float* params, const float* X, const float* mask, int32_t B,
                                         float* work, float* Y, int32_t* best, void* stream);

/* No counterpart in the reference (whose packing buffers are allocated inside
 * every call). For callers that cannot allocate device memory when they call:
 * a host application that owns the device memory budget and forbids its
 * plug-ins to call cudaMalloc, or a latency-critical loop that cannot afford
 * cudaMalloc/cudaFree and the synchronisation they may bring. Runs an FP32
 * plan (the SIMT kernel, any split_k) with the split-K scratch in a static
 * device array of MAXMULSK_STATIC_SCRATCH_BYTES that the library reserves on
 * every GPU that loads it, held until the process exits; nothing is
 * allocated. A plan needing more scratch returns MAXMULSK_ERR_UNSUPPORTED (C
 * untouched). The array is shared by every call on a device and keeps the last
 * call's contents: calls that overlap on the GPU race on it. The first call
 * on a device resolves the array's address with that device current; make it
 * before any stream capture. Asynchronous on `stream`. */
#define MAXMULSK_STATIC_SCRATCH_BYTES (16u << 20)
maxmulsk_status maxmulsk_sgemm_plan_static_dev(const float* dA, const float* dB, float* dC,
                                               size_t M, size_t K, size_t N,
                                               const maxmulsk_plan* plan, void* stream);

/* ----------------------------------------------------------------------------
 * FP64 checking (not on the product path: no GEMM entry point calls these).
 * The GPU form of the reference's FP64 checks (every library compared with an
 * FP64 product before timing, docs/BENCHMARKS.md:112-120 and :395-399) and of
 * its checker Utils::check_correctness (common/utils.hpp:24-48), for products
 * too large for a CPU loop in a test (4096^3, K = 32768, grouped batches).
 * ------------------------------------------------------------------------- */

/* C64[i][j] = sum_k (double)A[i][k] * (double)B[k][j], one fused multiply-add
 * chain per output over k in increasing order from +0 -- bit for bit the
 * sequential CPU loop (the product of two floats is exact in double). With
 * dCabs non-NULL, also Cabs[i][j] = sum_k |A[i][k]| |B[k][j]| the same way.
 * M x N doubles each, row-major. Asynchronous on `stream`. */
maxmulsk_status maxmulsk_check_dgemm_dev(const float* dA, const float* dB, double* dC64, double* dCabs,
                                         size_t M, size_t K, size_t N, void* stream);

/* Error measures of an FP32 result C against C64. */
typedef struct {
    double normwise;   /* ||C - C64||_F / (||A||_F ||B||_F)                     */
    double max_rel;    /* max |C - C64| / max(|C64|, 2^-24 Cabs), Cabs = 0 when
                          no dCabs is given                                     */
    double rel_frob;   /* ||C - C64||_F / ||C64||_F                             */
    double max_abs;    /* max |C - C64|                                         */
    double norm_a, norm_b, norm_diff, norm_c64;   /* the Frobenius norms used   */
} maxmulsk_error_report;

/* Bytes of device work memory maxmulsk_check_errors_dev needs (8-byte aligned). */
size_t maxmulsk_check_errors_work_bytes(void);

/* Computes the report with a deterministic two-pass reduction on the device
 * (a fixed number of blocks, each summing a fixed subset in a fixed order,
 * then the block results added in block order), waits for `stream` and writes
 * it to *out (host memory). dCabs may be NULL. */
maxmulsk_status maxmulsk_check_errors_dev(const float* dC, const double* dC64, const double* dCabs,
                                          const float* dA, const float* dB, size_t M, size_t K, size_t N,
                                          void* work, size_t work_bytes, maxmulsk_error_report* out,
                                          void* stream);

/* ----------------------------------------------------------------------------
 * Status, errors, device properties.
 * ------------------------------------------------------------------------- */

/* Waits for `stream` and returns MAXMULSK_ERR_TIMEOUT if any kernel of this
 * library on the current device gave up a bounded wait since the last call
 * (the flag is then cleared), MAXMULSK_ERR_CUDA on a CUDA error, else OK. */
maxmulsk_status maxmulsk_stream_status(void* stream);

/* A static, human-readable name for a status. */
const char* maxmulsk_status_string(maxmulsk_status s);

/* The text of the last CUDA error this thread saw inside the library. */
const char* maxmulsk_last_error_message(void);

/* Library version, e.g. "0.1.0". */
const char* maxmulsk_version(void);

/* ----------------------------------------------------------------------------
 * Phase timing: the counterpart of the reference's lab hooks
 * (sme/support/lab_hooks.hpp:1-22, scopes in
 * sme/v3/sme-1x4-acc-kcout.cpp:453-561) and of its per-phase timing breakdown
 * (sme/support/test_sme.cpp:580-678). Off by default; on with
 * MAXMULSK_PHASE_TIMING=1 in the environment or maxmulsk_phase_timing(1).
 * While on, every call outside a CUDA graph capture records a CUDA event pair
 * on its stream around each phase, and an NVTX range on the host thread:
 *   "split"   operand planes of the split-precision path (pre-pass)
 *   "gemm"    the GEMM kernel (SIMT or tcgen05)
 *   "reduce"  the split-K reduction kernel of plans with 3 or more K slices
 *   "grouped" one grouped batch (its CUDA graph)
 *   "h2d" / "d2h"  the host entry points' copies (pipelined copies overlap)
 * Up to 65536 phases are held between two reports; later ones are dropped.
 * ------------------------------------------------------------------------- */
void maxmulsk_phase_timing(int32_t on);

/* Waits for the phases recorded since the last report and writes
 * {"split": {"calls": n, "ms": t}, ...} (device milliseconds summed per phase;
 * phases with no calls omitted) into buf, NUL-terminated, truncated to len
 * bytes, and forgets them. Returns the length of the whole text, which never
 * exceeds MAXMULSK_PHASE_REPORT_BYTES - 1. */
#define MAXMULSK_PHASE_REPORT_BYTES 1024
size_t maxmulsk_phase_report(char* buf, size_t len);

#ifdef __cplusplus
}
#endif
