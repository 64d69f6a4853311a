// Learned cost model: a 2-hidden-layer MLP (64 GELU units each, FP32) that
// predicts the log-time of every candidate plan of a shape. Hand-written
// CUDA for training (forward, backward, Adam) and batched inference, plus a
// host forward pass with the same arithmetic order for the per-call picker.
//
// Counterpart in the reference: the hand-written shape rules and table it
// replaces (SMEKernels1x4V4C::choose, sme/v4/sme-1x4-v4c-dispatch.cpp:17-22;
// the v5.1 fixed plan, sme/v5/sme-1x4-fusedpack-v51.cpp:744-747; the tuning
// table, sme/support/gemm_tuning.cpp:34-37).
//
// Parameters are one flat FP32 array:
//   W1[F][H] b1[H] W2[H][H] b2[H] W3[H][O] b3[O]     (F = 7, H = 64, O = 48)
// Features of a shape (M, K, N, class):
//   ln(M), ln(N), ln(K) / ln(16384); (M, N, K mod 16) / 16; class (0 FP32, 1 split)
// Every kernel is deterministic: reductions run in a fixed order, no atomics.
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.hpp"
#include "mlp.hpp"
#include "runtime.hpp"

namespace mmsk {

namespace {

constexpr int F = MAXMULSK_MLP_FEATURES, H = MAXMULSK_MLP_HIDDEN, O = MAXMULSK_MLP_OUTPUTS;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + F * H, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H * O, NPARAM = OFF_B3 + O;
static_assert(NPARAM == MAXMULSK_MLP_PARAMS, "parameter count");

// GELU, exact form 0.5 x (1 + erf(x / sqrt 2)), and its derivative.
__host__ __device__ inline float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__host__ __device__ inline float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// Z[b][o] = b[o] + sum_i X[b][i] W[i][o]; A = act(Z) (GELU when act != 0).
__global__ void linear_fwd(const float* __restrict__ X, const float* __restrict__ W, const float* __restrict__ bias,
                           int B, int in, int out, float* __restrict__ Z, float* __restrict__ A, int act) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * out) return;
    const int b = idx / out, o = idx % out;
    float z = bias[o];
    for (int i = 0; i < in; i++) z = fmaf(X[b * in + i], W[i * out + o], z);
    if (Z) Z[idx] = z;
    if (A) A[idx] = act ? gelu(z) : z;
}

// dY = 2 (Y - T) / count over the entries with mask != 0 (else 0); the
// per-row squared errors go to rowloss[b] (summed on the host).
__global__ void mse_grad(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ mask,
                         int B, float inv_count, float* __restrict__ dY, float* __restrict__ rowloss) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    float l = 0.f;
    for (int o = 0; o < O; o++) {
        const int k = b * O + o;
        const float m = mask[k];
        const float d = (m != 0.f) ? (Y[k] - T[k]) : 0.f;
        dY[k] = 2.f * d * inv_count;
        l = fmaf(d, d, l);
    }
    rowloss[b] = l;
}

// dX[b][i] = sum_o dZ[b][o] W[i][o]; optionally times gelu'(Zprev[b][i]).
__global__ void linear_bwd_x(const float* __restrict__ dZ, const float* __restrict__ W, const float* __restrict__ Zprev,
                             int B, int in, int out, float* __restrict__ dX) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * in) return;
    const int b = idx / in, i = idx % in;
    float s = 0.f;
    for (int o = 0; o < out; o++) s = fmaf(dZ[b * out + o], W[i * out + o], s);
    dX[idx] = Zprev ? s * gelu_grad(Zprev[idx]) : s;
}

// dW[i][o] = sum_b X[b][i] dZ[b][o] (b upward), db[o] = sum_b dZ[b][o].
__global__ void linear_bwd_w(const float* __restrict__ X, const float* __restrict__ dZ, int B, int in, int out,
                             float* __restrict__ dW, float* __restrict__ db) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < in * out) {
        const int i = idx / out, o = idx % out;
        float s = 0.f;
        for (int b = 0; b < B; b++) s = fmaf(X[b * in + i], dZ[b * out + o], s);
        dW[idx] = s;
    } else if (idx < in * out + out) {
        const int o = idx - in * out;
        float s = 0.f;
        for (int b = 0; b < B; b++) s += dZ[b * out + o];
        db[o] = s;
    }
}

// Adam (bias-corrected), elementwise.
__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// best[b] = argmin over o with mask != 0 of Y[b][o] (lowest index on ties; -1 if none).
__global__ void masked_argmin(const float* __restrict__ Y, const float* __restrict__ mask, int B, int* __restrict__ best) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    int bi = -1;
    float bv = 0.f;
    for (int o = 0; o < O; o++) {
        if (mask[b * O + o] == 0.f) continue;
        const float y = Y[b * O + o];
        if (bi < 0 || y < bv) { bi = o; bv = y; }
    }
    best[b] = bi;
}

inline unsigned blocks(int n) { return (unsigned)((n + 255) / 256); }

// ----------------------------------------------------------------- host model
struct Model {
    bool loaded = false;
    std::vector<float> w;                     // NPARAM
};
std::mutex g_model_mu;
Model g_model;
bool g_env_tried = false;

void host_forward(const float* w, const float* x, float* y) {
    float h1[H], h2[H];
    for (int o = 0; o < H; o++) {
        float z = w[OFF_B1 + o];
        for (int i = 0; i < F; i++) z = fmaf(x[i], w[OFF_W1 + i * H + o], z);
        h1[o] = gelu(z);
    }
    for (int o = 0; o < H; o++) {
        float z = w[OFF_B2 + o];
        for (int i = 0; i < H; i++) z = fmaf(h1[i], w[OFF_W2 + i * H + o], z);
        h2[o] = gelu(z);
    }
    for (int o = 0; o < O; o++) {
        float z = w[OFF_B3 + o];
        for (int i = 0; i < H; i++) z = fmaf(h2[i], w[OFF_W3 + i * O + o], z);
        y[o] = z;
    }
}

// <directory of this library>/../data/picker_model.bin
std::string default_model_path() {
    Dl_info info;
    if (!dladdr(reinterpret_cast<void*>(&mlp_features), &info) || !info.dli_fname) return std::string();
    std::string so(info.dli_fname);
    const size_t slash = so.rfind('/');
    const std::string dir = (slash == std::string::npos) ? std::string(".") : so.substr(0, slash);
    return dir + "/../data/picker_model.bin";
}

bool load_file(const char* path, std::vector<float>& w) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char magic[8];
    int32_t dims[4];
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "MMSKMLP1", 8) == 0 &&
              std::fread(dims, sizeof(int32_t), 4, f) == 4 && dims[0] == F && dims[1] == H && dims[2] == O &&
              dims[3] == NPARAM;
    if (ok) {
        w.resize(NPARAM);
        ok = std::fread(w.data(), sizeof(float), NPARAM, f) == (size_t)NPARAM;
    }
    std::fclose(f);
    return ok;
}

}  // namespace

void mlp_features(size_t M, size_t K, size_t N, int cls, float* x) {
    const double s = 1.0 / std::log(16384.0);
    x[0] = (float)(std::log((double)(M ? M : 1)) * s);
    x[1] = (float)(std::log((double)(N ? N : 1)) * s);
    x[2] = (float)(std::log((double)(K ? K : 1)) * s);
    x[3] = (float)(M % 16) / 16.0f;
    x[4] = (float)(N % 16) / 16.0f;
    x[5] = (float)(K % 16) / 16.0f;
    x[6] = (float)cls;
}

int mlp_load(const char* path) {
    std::vector<float> w;
    if (!load_file(path, w)) return -1;
    std::lock_guard<std::mutex> lk(g_model_mu);
    g_env_tried = true;
    g_model.w = std::move(w);
    g_model.loaded = true;
    return 0;
}

void mlp_unload() {
    std::lock_guard<std::mutex> lk(g_model_mu);
    g_env_tried = true;
    g_model.loaded = false;
    g_model.w.clear();
}

bool mlp_predict_host(size_t M, size_t K, size_t N, int cls, float* y) {
    std::lock_guard<std::mutex> lk(g_model_mu);
    if (!g_env_tried) {
        // MAXMULSK_MODEL names the weights; unset, the model shipped beside
        // the library (data/picker_model.bin) is used if present; "" or
        // "none" runs without a model (the rule picks).
        g_env_tried = true;
        const char* env = std::getenv("MAXMULSK_MODEL");
        const std::string path = env ? std::string(env) : default_model_path();
        std::vector<float> w;
        if (!path.empty() && path != "none" && load_file(path.c_str(), w)) {
            g_model.w = std::move(w);
            g_model.loaded = true;
        }
    }
    if (!g_model.loaded) return false;
    float x[F];
    mlp_features(M, K, N, cls, x);
    host_forward(g_model.w.data(), x, y);
    return true;
}

bool mlp_predict_plan(size_t M, size_t K, size_t N, int precision, maxmulsk_plan* out, float* margin) {
    const int cls = (precision == MAXMULSK_PREC_FP32) ? 0 : 1;
    if (precision == MAXMULSK_PREC_BF16X9) return false;          // not among the candidates
    float y[O];
    if (!mlp_predict_host(M, K, N, cls, y)) return false;
    maxmulsk_plan cands[O];
    const int n = candidate_plans(cls, cands, O);
    const size_t max_workspace = (64u << 20) + 4 * sizeof(float) * (M * K + K * N + M * N);
    int best = -1, second = -1;
    for (int i = 0; i < n; i++) {
        if (precision != MAXMULSK_PREC_FP32 && precision != MAXMULSK_PREC_SPLIT_AUTO &&
            cands[i].precision != precision)
            continue;                                              // an explicit split mode
        if (classify_plan(M, K, N, &cands[i]) != MAXMULSK_OK) continue;
        // Plans with outsized split-K scratch were never timed (the autotuner
        // masks them), so the model's estimate for them means nothing.
        if (workspace_bytes(M, K, N, cands[i]) > max_workspace) continue;
        if (best < 0 || y[i] < y[best]) { second = best; best = i; }
        else if (second < 0 || y[i] < y[second]) second = i;
    }
    if (best < 0) return false;
    *out = cands[best];
    // Predicted log-time gap to the runner-up (infinite with one candidate).
    if (margin) *margin = second < 0 ? INFINITY : y[second] - y[best];
    return true;
}

}  // namespace mmsk

using namespace mmsk;

extern "C" {

maxmulsk_status maxmulsk_mlp_forward_dev(const float* params, const float* X, int32_t B, float* Z1, float* H1,
                                         float* Z2, float* H2, float* Y, void* stream) {
    if (!params || !X || !H1 || !H2 || !Y || B < 0) return MAXMULSK_ERR_INVALID;
    if (B == 0) return MAXMULSK_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    linear_fwd<<<blocks(B * H), 256, 0, s>>>(X, params + OFF_W1, params + OFF_B1, B, F, H, Z1, H1, 1);
    linear_fwd<<<blocks(B * H), 256, 0, s>>>(H1, params + OFF_W2, params + OFF_B2, B, H, H, Z2, H2, 1);
    linear_fwd<<<blocks(B * O), 256, 0, s>>>(H2, params + OFF_W3, params + OFF_B3, B, H, O, nullptr, Y, 0);
    return cuda_status(cudaGetLastError(), "mlp forward");
}

maxmulsk_status maxmulsk_mlp_backward_dev(const float* params, const float* X, const float* Z1, const float* H1,
                                          const float* Z2, const float* H2, const float* Y, const float* T,
                                          const float* mask, int32_t B, float count, float* grads, float* work,
                                          float* rowloss, void* stream) {
    if (!params || !X || !Z1 || !H1 || !Z2 || !H2 || !Y || !T || !mask || !grads || !work || !rowloss || B <= 0 ||
        !(count > 0))
        return MAXMULSK_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float* dY = work;                    // B x O
    float* dZ2 = dY + (size_t)B * O;     // B x H
    float* dZ1 = dZ2 + (size_t)B * H;    // B x H
    mse_grad<<<blocks(B), 256, 0, s>>>(Y, T, mask, B, 1.0f / count, dY, rowloss);
    linear_bwd_w<<<blocks(H * O + O), 256, 0, s>>>(H2, dY, B, H, O, grads + OFF_W3, grads + OFF_B3);
    linear_bwd_x<<<blocks(B * H), 256, 0, s>>>(dY, params + OFF_W3, Z2, B, H, O, dZ2);
    linear_bwd_w<<<blocks(H * H + H), 256, 0, s>>>(H1, dZ2, B, H, H, grads + OFF_W2, grads + OFF_B2);
    linear_bwd_x<<<blocks(B * H), 256, 0, s>>>(dZ2, params + OFF_W2, Z1, B, H, H, dZ1);
    linear_bwd_w<<<blocks(F * H + H), 256, 0, s>>>(X, dZ1, B, F, H, grads + OFF_W1, grads + OFF_B1);
    return cuda_status(cudaGetLastError(), "mlp backward");
}

maxmulsk_status maxmulsk_mlp_adam_dev(float* params, const float* grads, float* m, float* v, float lr, float beta1,
                                      float beta2, float eps, int32_t step, void* stream) {
    if (!params || !grads || !m || !v || step < 1) return MAXMULSK_ERR_INVALID;
    const float c1 = 1.0f - std::pow(beta1, (float)step), c2 = 1.0f - std::pow(beta2, (float)step);
    adam_step<<<blocks(NPARAM), 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grads, m, v, NPARAM, lr, beta1,
                                                                              beta2, eps, c1, c2);
    return cuda_status(cudaGetLastError(), "mlp adam");
}

maxmulsk_status maxmulsk_mlp_predict_dev(const float* params, const float* X, const float* mask, int32_t B,
                                         float* work, float* Y, int32_t* best, void* stream) {
    if (!params || !X || !Y || !work || B < 0) return MAXMULSK_ERR_INVALID;
    if (B == 0) return MAXMULSK_OK;
    float* H1 = work;
    float* H2 = work + (size_t)B * H;
    maxmulsk_status st = maxmulsk_mlp_forward_dev(params, X, B, nullptr, H1, nullptr, H2, Y, stream);
    if (st != MAXMULSK_OK) return st;
    if (best && mask) {
        masked_argmin<<<blocks(B), 256, 0, static_cast<cudaStream_t>(stream)>>>(Y, mask, B, best);
        return cuda_status(cudaGetLastError(), "mlp argmin");
    }
    return MAXMULSK_OK;
}

maxmulsk_status maxmulsk_mlp_features(size_t M, size_t K, size_t N, int32_t cls, float* out) {
    if (!out) return MAXMULSK_ERR_INVALID;
    mlp_features(M, K, N, cls, out);
    return MAXMULSK_OK;
}

maxmulsk_status maxmulsk_mlp_predict_host(size_t M, size_t K, size_t N, int32_t cls, float* out) {
    if (!out) return MAXMULSK_ERR_INVALID;
    return mlp_predict_host(M, K, N, cls, out) ? MAXMULSK_OK : MAXMULSK_ERR_UNSUPPORTED;
}

maxmulsk_status maxmulsk_model_load(const char* path) {
    if (!path) { mlp_unload(); return MAXMULSK_OK; }
    return mlp_load(path) == 0 ? MAXMULSK_OK : MAXMULSK_ERR_INVALID;
}

}  // extern "C"
