// Exhaustive autotuner over a fixed candidate list.
//
// The reference tunes by hand: sweeps run in its Lab harness
// (bench/results/2026-09-13/source/RERUN.txt:13-16, 100 blockings x 35 shapes),
// and only results that held across three runs became table entries
// (sme/support/gemm_tuning.hpp:8-24). Here every candidate of a shape is
// timed on the device: each one is warmed once, then a CUDA graph of `reps`
// calls is replayed three times and the median replay gives the time per
// call, so host launch gaps never enter the measurement.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.hpp"
#include "mlp.hpp"
#include "phase.hpp"
#include "runtime.hpp"
#include "tuning.hpp"

namespace mmsk {

int candidate_plans(int cls, maxmulsk_plan* out, int cap) {
    int n = 0;
    auto add = [&](int prec, int tm, int tn, int sk, int variant = 0) {
        if (n >= cap) return;
        maxmulsk_plan p;
        std::memset(&p, 0, sizeof p);
        p.precision = prec; p.tile_m = tm; p.tile_n = tn; p.split_k = sk; p.variant = variant;
        out[n++] = p;
    };
    if (cls == 0) {
        const int tiles[3][2] = {{128, 128}, {128, 64}, {64, 64}};
        const int splits[8] = {1, 2, 4, 8, 16, 24, 32, 64};
        for (auto& t : tiles)
            for (int sk : splits) add(MAXMULSK_PREC_FP32, t[0], t[1], sk);
    } else {
        // 18 + 18 planes-in-memory plans, 7 fused-split plans (narrow shapes
        // need deep K splits; split 0 fills the SMs with one K slice per
        // slot), 5 narrow-tile plans: 48.
        const int modes[2] = {MAXMULSK_PREC_3XTF32, MAXMULSK_PREC_BF16X6};
        const int tiles[3][2] = {{128, 128}, {128, 256}, {256, 256}};
        const int splits[6] = {1, 2, 4, 8, 16, 32};
        for (int m : modes)
            for (auto& t : tiles)
                for (int sk : splits) add(m, t[0], t[1], sk);
        const int fused_splits[7] = {1, 2, 4, 8, 16, 32, 0};
        for (int sk : fused_splits) add(MAXMULSK_PREC_BF16X6, 128, 128, sk, MAXMULSK_TC_FUSED_SPLIT);
        add(MAXMULSK_PREC_3XTF32, 128, 64, 4);
        add(MAXMULSK_PREC_3XTF32, 128, 64, 16);
        add(MAXMULSK_PREC_BF16X6, 128, 64, 1);
        add(MAXMULSK_PREC_BF16X6, 128, 64, 4);
        add(MAXMULSK_PREC_BF16X6, 128, 64, 16);
    }
    return n;
}

namespace {

struct TuneStream {
    cudaStream_t s = nullptr;
    ~TuneStream() { if (s) cudaStreamDestroy(s); }
};
thread_local TuneStream t_tune;

// Median per-call time of `plan` in microseconds, or +inf if it cannot run.
maxmulsk_status time_plan(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                          const maxmulsk_plan& plan, void* ws, size_t ws_bytes, int reps, float* out) {
    *out = INFINITY;
    if (classify_plan(M, K, N, &plan) != MAXMULSK_OK) return MAXMULSK_OK;
    if (workspace_bytes(M, K, N, plan) > ws_bytes) return MAXMULSK_OK;
    if (!t_tune.s) {
        maxmulsk_status st = cuda_status(cudaStreamCreateWithFlags(&t_tune.s, cudaStreamNonBlocking), "stream");
        if (st != MAXMULSK_OK) return st;
    }
    cudaStream_t s = t_tune.s;
    PhaseMute mute;                                  // timing runs are not the caller's phases
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    maxmulsk_status st = run_plan_dev(dA, dB, dC, M, K, N, plan, ws, ws_bytes, s);   // warm-up
    if (st == MAXMULSK_OK) st = stream_status(s);
    if (st != MAXMULSK_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return st; }
    if (reps <= 0) {
        cudaEventRecord(e0, s);
        run_plan_dev(dA, dB, dC, M, K, N, plan, ws, ws_bytes, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        reps = (int)std::min(64.0, std::max(1.0, std::ceil(0.5 / std::max(1e-4, (double)ms))));
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int r = 0; r < reps && st == MAXMULSK_OK; r++) st = run_plan_dev(dA, dB, dC, M, K, N, plan, ws, ws_bytes, s);
        cudaError_t e2 = cudaStreamEndCapture(s, &graph);
        if (e == cudaSuccess) e = e2;
    }
    if (e == cudaSuccess && st == MAXMULSK_OK) e = cudaGraphInstantiate(&exec, graph, 0);
    float t[3] = {INFINITY, INFINITY, INFINITY};
    if (e == cudaSuccess && st == MAXMULSK_OK) {
        e = cudaGraphLaunch(exec, s);                                // warm the graph
        for (int i = 0; i < 3 && e == cudaSuccess; i++) {
            cudaEventRecord(e0, s);
            e = cudaGraphLaunch(exec, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            t[i] = ms * 1000.f / (float)reps;
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MAXMULSK_OK) return st;
    if (e != cudaSuccess) return cuda_status(e, "autotune graph");
    st = stream_status(s);
    if (st != MAXMULSK_OK) return st;
    std::sort(t, t + 3);
    *out = t[1];
    return MAXMULSK_OK;
}

}  // namespace

void autotune_fallback(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N, int precision,
                       cudaStream_t s) {
    if (M == 0 || N == 0 || K == 0 || !dA || !dB || !dC) return;
    if (!autotune_fallback_enabled() || !picker_doubt(M, K, N, precision)) return;
    // Never inside a stream capture: the search synchronises and times.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) { cudaGetLastError(); return; }
    if (cs != cudaStreamCaptureStatusNone) return;
    // Workspace for every candidate the learned model would also consider
    // (split-K scratch up to 64 MiB + 4x the operand bytes).
    const int cls = precision == MAXMULSK_PREC_FP32 ? 0 : 1;
    maxmulsk_plan cands[MAXMULSK_MLP_OUTPUTS];
    const int n = candidate_plans(cls, cands, MAXMULSK_MLP_OUTPUTS);
    const size_t cap = (64u << 20) + 4 * sizeof(float) * (M * K + K * N + M * N);
    size_t need = 0;
    for (int i = 0; i < n; i++) {
        if (classify_plan(M, K, N, &cands[i]) != MAXMULSK_OK) continue;
        const size_t w = workspace_bytes(M, K, N, cands[i]);
        if (w <= cap && w > need) need = w;
    }
    maxmulsk_status st = MAXMULSK_OK;
    size_t ws_bytes = 0;
    void* ws = need ? managed_workspace(s, need, &ws_bytes, &st) : nullptr;
    if (need && !ws) return;
    maxmulsk_plan best;
    float us = 0.f;
    st = maxmulsk_autotune_dev(dA, dB, dC, M, K, N, precision, ws, ws_bytes, &best, &us, s);
    (void)st;   // on failure the picker keeps to the model or the rule
}

}  // namespace mmsk

using namespace mmsk;

extern "C" {

size_t maxmulsk_candidates(int32_t cls, maxmulsk_plan* out, size_t cap) {
    if (cls != 0 && cls != 1) return 0;
    maxmulsk_plan tmp[MAXMULSK_MLP_OUTPUTS];
    const int n = candidate_plans(cls, tmp, MAXMULSK_MLP_OUTPUTS);
    const size_t k = std::min((size_t)n, out ? cap : 0);
    for (size_t i = 0; i < k; i++) out[i] = tmp[i];
    return out ? k : (size_t)n;
}

maxmulsk_status maxmulsk_autotune_time_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                           const maxmulsk_plan* plans, size_t nplans, void* ws, size_t ws_bytes,
                                           int32_t reps, float* times_us, void* stream) {
    if (!plans || !times_us) return MAXMULSK_ERR_INVALID;
    maxmulsk_status st = cuda_status(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "sync");
    if (st != MAXMULSK_OK) return st;
    for (size_t i = 0; i < nplans; i++) {
        st = time_plan(dA, dB, dC, M, K, N, plans[i], ws, ws_bytes, reps, &times_us[i]);
        if (st != MAXMULSK_OK) return st;
    }
    return MAXMULSK_OK;
}

maxmulsk_status maxmulsk_autotune_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                      int32_t precision, void* ws, size_t ws_bytes, maxmulsk_plan* best,
                                      float* best_us, void* stream) {
    if (precision < MAXMULSK_PREC_FP32 || precision > MAXMULSK_PREC_SPLIT_AUTO || precision == MAXMULSK_PREC_BF16X9)
        return MAXMULSK_ERR_UNSUPPORTED;
    const int cls = precision == MAXMULSK_PREC_FP32 ? 0 : 1;
    maxmulsk_plan cands[MAXMULSK_MLP_OUTPUTS];
    const int n = candidate_plans(cls, cands, MAXMULSK_MLP_OUTPUTS);
    std::vector<maxmulsk_plan> use;
    for (int i = 0; i < n; i++)
        if (precision == MAXMULSK_PREC_FP32 || precision == MAXMULSK_PREC_SPLIT_AUTO || cands[i].precision == precision)
            use.push_back(cands[i]);
    std::vector<float> t(use.size(), INFINITY);
    maxmulsk_status st = maxmulsk_autotune_time_dev(dA, dB, dC, M, K, N, use.data(), use.size(), ws, ws_bytes, 0,
                                                    t.data(), stream);
    if (st != MAXMULSK_OK) return st;
    size_t bi = 0;
    for (size_t i = 1; i < t.size(); i++)
        if (t[i] < t[bi]) bi = i;
    if (!(t[bi] < INFINITY)) { set_error_message("no candidate could run"); return MAXMULSK_ERR_UNSUPPORTED; }
    tuning_put(M, K, N, precision, use[bi], t[bi]);
    if (best) *best = use[bi];
    if (best_us) *best_us = t[bi];
    return MAXMULSK_OK;
}

}  // extern "C"
