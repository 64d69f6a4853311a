// Plans: validation, workspace sizing, the fixed shape rule and the tuned
// picker with its environment override.
//
// Counterparts in the reference:
//   classify_plan   NB::classify   sme/v4/sme-1x4-kcout-ncblock-apack4za.cpp:410-423
//   workspace_bytes NB::capacity   :429-444, v5.1 workspace_bytes (sme/v5/sme-1x4-fusedpack-v51.hpp:75-78)
//   choose_rule     SMEKernels1x4V4C::choose  sme/v4/sme-1x4-v4c-dispatch.cpp:17-22
//   choose_tuned    MaxMulSK::tuning::select  sme/support/gemm_tuning.cpp:96-100
//   parse_config_env parse_env(MAXMULSK_BLOCKING)  sme/support/gemm_tuning.cpp:66-78
//   picker_doubt    when the learned model is not to be trusted and the
//                   exhaustive search (autotune.cpp) runs instead; the
//                   reference's counterpart is the MAXMULSK_BLOCKING sweep
//                   that overrides its table (gemm_tuning.cpp:66-78, 96-100)
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "internal.hpp"
#include "mlp.hpp"
#include "runtime.hpp"
#include "tuning.hpp"

namespace mmsk {

namespace {
bool is_tc(int precision) {
    return precision == MAXMULSK_PREC_3XTF32 || precision == MAXMULSK_PREC_BF16X6 ||
           precision == MAXMULSK_PREC_BF16X9;
}
constexpr size_t kMaxDim = 0x7FFFFFFFull;   // TMA coordinates and grid sizes are 32-bit
}  // namespace

maxmulsk_status classify_plan(size_t M, size_t K, size_t N, const maxmulsk_plan* plan) {
    if (!plan) { set_error_message("null plan"); return MAXMULSK_ERR_INVALID; }
    const maxmulsk_plan& p = *plan;
    if (p.split_k < 0 || p.split_k > 64 || (p.split_k == 0 && p.precision == MAXMULSK_PREC_FP32)) {
        set_error_message("split_k must be 1..64 (0: fill the SMs, tensor-core plans only)");
        return MAXMULSK_ERR_UNSUPPORTED;
    }
    if (p.precision == MAXMULSK_PREC_FP32) {
        const bool tile_ok = (p.tile_m == 128 && p.tile_n == 128) || (p.tile_m == 128 && p.tile_n == 64) ||
                             (p.tile_m == 64 && p.tile_n == 64);
        if (!tile_ok) { set_error_message("FP32 tiles: 128x128, 128x64 or 64x64"); return MAXMULSK_ERR_UNSUPPORTED; }
        if (p.variant != MAXMULSK_FP32_FMA && p.variant != MAXMULSK_FP32_SCALAR) {
            set_error_message("unknown FP32 variant");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
        if (M > kMaxDim || N > kMaxDim || K > kMaxDim) { set_error_message("dimension too large"); return MAXMULSK_ERR_UNSUPPORTED; }
        if ((M + p.tile_m - 1) / p.tile_m > 65535) { set_error_message("M too large for the FP32 grid"); return MAXMULSK_ERR_UNSUPPORTED; }
        if (p.chunk != 0) { set_error_message("FP32 plans take chunk 0"); return MAXMULSK_ERR_UNSUPPORTED; }
        return MAXMULSK_OK;
    }
    if (is_tc(p.precision)) {
        const bool single = p.tile_m == 128 && (p.tile_n == 64 || p.tile_n == 128 || p.tile_n == 256);
        const bool pair = p.tile_m == 256 && (p.tile_n == 128 || p.tile_n == 256);
        if (!single && !pair) {
            set_error_message("tensor-core tiles: 128x64, 128x128, 128x256 (one CTA), 256x128, 256x256 (CTA pair)");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
        if (p.variant != MAXMULSK_TC_SPLIT_INPUTS && p.variant != MAXMULSK_TC_REUSE_PLANES &&
            p.variant != MAXMULSK_TC_FUSED_SPLIT) {
            set_error_message("unknown tensor-core variant");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
        if (p.variant == MAXMULSK_TC_FUSED_SPLIT &&
            (p.precision == MAXMULSK_PREC_3XTF32 || p.tile_m != 128 || p.tile_n != 128 || K % 4 != 0 || N % 4 != 0)) {
            set_error_message("the fused split runs BF16X6 / BF16X9 on 128x128 tiles with K and N multiples of 4");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
        if (M > kMaxDim || N > kMaxDim || K > kMaxDim) { set_error_message("dimension too large"); return MAXMULSK_ERR_UNSUPPORTED; }
        if (N > 32ull * 65535ull) { set_error_message("N too large for the split pre-pass grid"); return MAXMULSK_ERR_UNSUPPORTED; }
        if (p.chunk != 0 && (p.chunk < 32 || p.chunk > 4096 || p.chunk % 32 != 0)) {
            set_error_message("chunk must be 0 or a multiple of 32 in 32 .. 4096");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
        return MAXMULSK_OK;
    }
    set_error_message("unknown precision");
    return MAXMULSK_ERR_UNSUPPORTED;
}

size_t workspace_bytes(size_t M, size_t K, size_t N, const maxmulsk_plan& p) {
    if (M == 0 || N == 0 || K == 0) return 0;
    if (p.precision == MAXMULSK_PREC_FP32)
        return simt_workspace_bytes((int64_t)M, (int64_t)K, (int64_t)N, p.tile_m, p.tile_n, p.split_k);
    return tc_workspace_bytes((int64_t)M, (int64_t)K, (int64_t)N, p.precision, p.tile_m, p.tile_n, p.split_k);
}

// Two fixed profiles per precision, separated by shape alone, like the v4c
// rule. A large profile when the output alone fills the machine; otherwise a
// small tile with K cut into slices until roughly two waves of CTAs exist.
maxmulsk_plan choose_rule(size_t M, size_t K, size_t N, int precision, int sms) {
    maxmulsk_plan p;
    std::memset(&p, 0, sizeof(p));
    if (precision == MAXMULSK_PREC_SPLIT_AUTO) precision = MAXMULSK_PREC_3XTF32;
    p.precision = precision;
    p.split_k = 1;
    if (sms <= 0) sms = 148;
    if (precision == MAXMULSK_PREC_FP32) {
        const size_t big_tiles = ((M + 127) / 128) * ((N + 127) / 128);
        if (big_tiles >= (size_t)sms) {
            p.tile_m = 128; p.tile_n = 128;
        } else {
            p.tile_m = 64; p.tile_n = 64;
            const size_t tiles = ((M + 63) / 64) * ((N + 63) / 64);
            size_t want = (2 * (size_t)sms + tiles - 1) / tiles;
            const size_t kmax = K / 256 ? K / 256 : 1;          // keep slices >= 256 deep
            if (want > kmax) want = kmax;
            if (want > 64) want = 64;
            p.split_k = (int)(want ? want : 1);
        }
        return p;
    }
    p.tile_m = 128;
    const size_t t256 = ((M + 127) / 128) * ((N + 255) / 256);
    const size_t t128 = ((M + 127) / 128) * ((N + 127) / 128);
    size_t tiles;
    if (t256 >= (size_t)sms && N >= 256) { p.tile_n = 256; tiles = t256; }
    else { p.tile_n = 128; tiles = t128; }
    if (tiles < (size_t)sms) {
        size_t want = ((size_t)sms + tiles - 1) / tiles;
        const size_t kmax = K / 512 ? K / 512 : 1;
        if (want > kmax) want = kmax;
        if (want > 64) want = 64;
        p.split_k = (int)(want ? want : 1);
    }
    return p;
}

// MAXMULSK_CONFIG="precision,tile_m,tile_n,split_k[,variant[,chunk]]" overrides the
// picker; malformed values are ignored, as the reference's parse_env does.
bool parse_config_env(maxmulsk_plan& out) {
    const char* s = std::getenv("MAXMULSK_CONFIG");
    if (!s || !*s) return false;
    int prec = 0, tm = 0, tn = 0, sk = 0, var = 0, chunk = 0;
    const int n = std::sscanf(s, "%d,%d,%d,%d,%d,%d", &prec, &tm, &tn, &sk, &var, &chunk);
    if (n < 4) return false;
    if (tm <= 0 || tn <= 0 || sk <= 0 || chunk < 0) return false;
    maxmulsk_plan p;
    std::memset(&p, 0, sizeof(p));
    p.precision = prec; p.tile_m = tm; p.tile_n = tn; p.split_k = sk; p.variant = (n >= 5) ? var : 0;
    p.chunk = (n >= 6) ? chunk : 0;
    out = p;
    return true;
}

// Tuning database entry for this exact shape, else the learned cost model,
// else the rule. BF16X9 has no candidates or model class of its own: it
// takes the model's BF16X6 plan for the shape (the same tiles, K splits and
// variants run the nine products per k instead of six; the accuracy bar is
// asserted for every such plan).
maxmulsk_plan choose_tuned(size_t M, size_t K, size_t N, int precision, int sms) {
    maxmulsk_plan p;
    if (tuning_lookup(M, K, N, precision, &p)) return p;
    const int model_precision = precision == MAXMULSK_PREC_BF16X9 ? MAXMULSK_PREC_BF16X6 : precision;
    if (tuning_predict(M, K, N, model_precision, &p)) {
        if (precision == MAXMULSK_PREC_BF16X9) p.precision = MAXMULSK_PREC_BF16X9;
        return p;
    }
    return choose_rule(M, K, N, precision, sms);
}

namespace {
// The learned model was trained on M, N, K in [1, 16384].
constexpr size_t kTrainedMaxDim = 16384;

double env_double(const char* name, double dflt) {
    const char* s = std::getenv(name);
    if (!s || !*s) return dflt;
    char* end = nullptr;
    const double v = std::strtod(s, &end);
    return (end && *end == '\0') ? v : dflt;
}
}  // namespace

bool autotune_fallback_enabled() {
    const char* s = std::getenv("MAXMULSK_AUTOTUNE");
    return !(s && std::strcmp(s, "0") == 0);
}

const char* picker_doubt(size_t M, size_t K, size_t N, int precision) {
    // BF16X9 has no candidates of its own: the autotuner does not search it.
    if (precision == MAXMULSK_PREC_BF16X9) return nullptr;
    maxmulsk_plan p;
    if (tuning_lookup(M, K, N, precision, &p)) return nullptr;
    float margin = 0.f;
    if (!mlp_predict_plan(M, K, N, precision, &p, &margin)) return "no learned model";
    if (M > kTrainedMaxDim || N > kTrainedMaxDim || K > kTrainedMaxDim) return "shape outside the trained range";
    // Predicted ln-time gap to the runner-up. Measured on the committed
    // held-out timings, the gap barely predicts the model's regret (FP32:
    // 1.8 % mean regret below 0.005, 2.3 % above), so the search pays in
    // proportion to how often it runs; the default 0.005 sends about a sixth
    // of new shapes to it.
    if ((double)margin < env_double("MAXMULSK_AUTOTUNE_MARGIN", 0.005)) return "close call";
    return nullptr;
}

}  // namespace mmsk
