// The C ABI (include/maxmulsk.h). Thin: argument checks, the reference's
// empty-shape contract, plan selection, then the runtime.
//
// Reference counterpart: capi/maxmulsk.cpp:13-44 (handle_empty, to_status,
// maxmulsk_sgemm_v3, maxmulsk_sgemm_v4).
#include <cstring>

#include "maxmulsk.h"
#include "internal.hpp"
#include "phase.hpp"
#include "runtime.hpp"
#include "tuning.hpp"

namespace {

int sms_now() { return mmsk::device_sm_count(); }

// v3: the picker, FP32 SIMT; MAXMULSK_CONFIG wins. The picker: the tuning
// database, else -- when the learned model cannot be trusted for the shape
// (mmsk::picker_doubt) -- an exhaustive search on the call's own operands
// whose winner enters the database, else the model, else the rule. The
// search runs on device operands (dA, dB given, C overwritten), or, for host
// pointers, on device copies of A and B.
maxmulsk_plan plan_v3_host(const float* A, const float* B, size_t M, size_t K, size_t N) {
    maxmulsk_plan p;
    if (mmsk::parse_config_env(p)) return p;
    mmsk::autotune_fallback_host(A, B, M, K, N, MAXMULSK_PREC_FP32);
    return mmsk::choose_tuned(M, K, N, MAXMULSK_PREC_FP32, sms_now());
}
maxmulsk_plan plan_v3_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                          cudaStream_t s) {
    maxmulsk_plan p;
    if (mmsk::parse_config_env(p)) return p;
    mmsk::autotune_fallback(dA, dB, dC, M, K, N, MAXMULSK_PREC_FP32, s);
    return mmsk::choose_tuned(M, K, N, MAXMULSK_PREC_FP32, sms_now());
}

// v4: the fixed rule only.
maxmulsk_plan plan_v4(size_t M, size_t K, size_t N) {
    return mmsk::choose_rule(M, K, N, MAXMULSK_PREC_FP32, sms_now());
}

bool is_split_precision(int32_t prec) {
    return prec == MAXMULSK_PREC_3XTF32 || prec == MAXMULSK_PREC_BF16X6 || prec == MAXMULSK_PREC_BF16X9 ||
           prec == MAXMULSK_PREC_SPLIT_AUTO;
}

maxmulsk_plan plan_split_host(const float* A, const float* B, size_t M, size_t K, size_t N, int32_t prec) {
    maxmulsk_plan p;
    if (mmsk::parse_config_env(p) && p.precision == prec) return p;
    mmsk::autotune_fallback_host(A, B, M, K, N, prec);
    return mmsk::choose_tuned(M, K, N, prec, sms_now());
}
maxmulsk_plan plan_split_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N, int32_t prec,
                             cudaStream_t s) {
    maxmulsk_plan p;
    if (mmsk::parse_config_env(p) && p.precision == prec) return p;
    mmsk::autotune_fallback(dA, dB, dC, M, K, N, prec, s);
    return mmsk::choose_tuned(M, K, N, prec, sms_now());
}

}  // namespace

extern "C" {

maxmulsk_status maxmulsk_sgemm_v3(const float* A, const float* B, float* C, size_t M, size_t K, size_t N) {
    if (M == 0 || N == 0) return MAXMULSK_OK;
    return mmsk::run_plan_host(A, B, C, M, K, N, plan_v3_host(A, B, M, K, N));
}

maxmulsk_status maxmulsk_sgemm_v4(const float* A, const float* B, float* C, size_t M, size_t K, size_t N) {
    if (M == 0 || N == 0) return MAXMULSK_OK;
    return mmsk::run_plan_host(A, B, C, M, K, N, plan_v4(M, K, N));
}

maxmulsk_status maxmulsk_sgemm_v3_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                      void* stream) {
    if (M == 0 || N == 0) return MAXMULSK_OK;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return mmsk::run_plan_managed(dA, dB, dC, M, K, N, plan_v3_dev(dA, dB, dC, M, K, N, s), s);
}

maxmulsk_status maxmulsk_sgemm_v4_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                      void* stream) {
    if (M == 0 || N == 0) return MAXMULSK_OK;
    return mmsk::run_plan_managed(dA, dB, dC, M, K, N, plan_v4(M, K, N), static_cast<cudaStream_t>(stream));
}

maxmulsk_status maxmulsk_classify(size_t M, size_t K, size_t N, const maxmulsk_plan* plan) {
    return mmsk::classify_plan(M, K, N, plan);
}

maxmulsk_status maxmulsk_choose(size_t M, size_t K, size_t N, int32_t precision, maxmulsk_plan* out) {
    if (!out) return MAXMULSK_ERR_INVALID;
    if (precision != MAXMULSK_PREC_FP32 && !is_split_precision(precision)) return MAXMULSK_ERR_UNSUPPORTED;
    maxmulsk_plan p;
    if (mmsk::parse_config_env(p) && p.precision == precision) { *out = p; return MAXMULSK_OK; }
    *out = mmsk::choose_tuned(M, K, N, precision, sms_now());
    return MAXMULSK_OK;
}

const char* maxmulsk_picker_doubt(size_t M, size_t K, size_t N, int32_t precision) {
    if (precision != MAXMULSK_PREC_FP32 && !is_split_precision(precision)) return nullptr;
    if (!mmsk::autotune_fallback_enabled()) return nullptr;
    return mmsk::picker_doubt(M, K, N, precision);
}

maxmulsk_status maxmulsk_choose_rule(size_t M, size_t K, size_t N, int32_t precision, maxmulsk_plan* out) {
    if (!out) return MAXMULSK_ERR_INVALID;
    if (precision != MAXMULSK_PREC_FP32 && !is_split_precision(precision)) return MAXMULSK_ERR_UNSUPPORTED;
    *out = mmsk::choose_rule(M, K, N, precision, sms_now());
    return MAXMULSK_OK;
}

size_t maxmulsk_workspace_bytes(size_t M, size_t K, size_t N, const maxmulsk_plan* plan) {
    if (!plan || mmsk::classify_plan(M, K, N, plan) != MAXMULSK_OK) return 0;
    return mmsk::workspace_bytes(M, K, N, *plan);
}

maxmulsk_status maxmulsk_sgemm_plan_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                        const maxmulsk_plan* plan, void* ws, size_t ws_bytes, void* stream) {
    maxmulsk_status st = mmsk::classify_plan(M, K, N, plan);
    if (st != MAXMULSK_OK) return st;
    return mmsk::run_plan_dev(dA, dB, dC, M, K, N, *plan, ws, ws_bytes, static_cast<cudaStream_t>(stream));
}

maxmulsk_status maxmulsk_sgemm_plan(const float* A, const float* B, float* C, size_t M, size_t K, size_t N,
                                    const maxmulsk_plan* plan) {
    maxmulsk_status st = mmsk::classify_plan(M, K, N, plan);
    if (st != MAXMULSK_OK) return st;
    return mmsk::run_plan_host(A, B, C, M, K, N, *plan);
}

maxmulsk_status maxmulsk_sgemm_split(const float* A, const float* B, float* C, size_t M, size_t K, size_t N,
                                     int32_t precision) {
    if (!is_split_precision(precision)) return MAXMULSK_ERR_UNSUPPORTED;
    if (M == 0 || N == 0) return MAXMULSK_OK;
    return mmsk::run_plan_host(A, B, C, M, K, N, plan_split_host(A, B, M, K, N, precision));
}

maxmulsk_status maxmulsk_sgemm_split_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                         int32_t precision, void* stream) {
    if (!is_split_precision(precision)) return MAXMULSK_ERR_UNSUPPORTED;
    if (M == 0 || N == 0) return MAXMULSK_OK;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return mmsk::run_plan_managed(dA, dB, dC, M, K, N, plan_split_dev(dA, dB, dC, M, K, N, precision, s), s);
}

maxmulsk_status maxmulsk_sgemm_plan_static_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K,
                                               size_t N, const maxmulsk_plan* plan, void* stream) {
    if (!plan) { mmsk::set_error_message("null plan"); return MAXMULSK_ERR_INVALID; }
    return mmsk::simt_run_static_scratch(dA, dB, dC, M, K, N, *plan, static_cast<cudaStream_t>(stream));
}

void maxmulsk_phase_timing(int32_t on) { mmsk::phase_set(on != 0); }

size_t maxmulsk_phase_report(char* buf, size_t len) { return mmsk::phase_report(buf, len); }

size_t maxmulsk_probe_split_bytes(size_t R, size_t C, int32_t precision, int32_t as_b) {
    if (!is_split_precision(precision)) return 0;
    return mmsk::split_one_bytes((int64_t)R, (int64_t)C, precision, as_b != 0);
}

maxmulsk_status maxmulsk_probe_split_dev(const float* dX, size_t R, size_t C, int32_t precision, int32_t as_b,
                                         void* out, void* stream) {
    if (!is_split_precision(precision)) return MAXMULSK_ERR_UNSUPPORTED;
    if (R == 0 || C == 0) return MAXMULSK_OK;
    if (!dX || !out) return MAXMULSK_ERR_INVALID;
    return mmsk::cuda_status(mmsk::split_one(dX, (int64_t)R, (int64_t)C, precision, as_b != 0, out,
                                             static_cast<cudaStream_t>(stream)),
                             "split pre-pass launch");
}

maxmulsk_status maxmulsk_probe_timeout_dev(int64_t cycles, void* stream) {
    if (cycles <= 0 || cycles > 2000000000LL) { mmsk::set_error_message("cycles must be 1 .. 2e9"); return MAXMULSK_ERR_INVALID; }
    int* err = mmsk::device_error_word();
    if (!err) { mmsk::set_error_message("device error word unavailable"); return MAXMULSK_ERR_ALLOC; }
    return mmsk::cuda_status(mmsk::tc_timeout_probe(err, (long long)cycles, static_cast<cudaStream_t>(stream)),
                             "timeout probe launch");
}

maxmulsk_status maxmulsk_stream_status(void* stream) {
    return mmsk::stream_status(static_cast<cudaStream_t>(stream));
}

const char* maxmulsk_status_string(maxmulsk_status s) {
    switch (s) {
        case MAXMULSK_OK: return "MAXMULSK_OK";
        case MAXMULSK_ERR_UNSUPPORTED: return "MAXMULSK_ERR_UNSUPPORTED";
        case MAXMULSK_ERR_ALLOC: return "MAXMULSK_ERR_ALLOC";
        case MAXMULSK_ERR_CUDA: return "MAXMULSK_ERR_CUDA";
        case MAXMULSK_ERR_INVALID: return "MAXMULSK_ERR_INVALID";
        case MAXMULSK_ERR_TIMEOUT: return "MAXMULSK_ERR_TIMEOUT";
    }
    return "MAXMULSK_ERR_UNKNOWN";
}

const char* maxmulsk_last_error_message(void) { return mmsk::last_error_message(); }

const char* maxmulsk_version(void) { return "0.1.0"; }

}  // extern "C"
