// Host runtime: device state, workspace cache, host staging and dispatch.
//
// The reference allocates its packing buffers inside every call and frees
// them on return (sme/v3/sme-1x4-acc-kcout.cpp:455-461,
// sme/v4/sme-1x4-kcout-ncblock-apack4za.cpp:638-654). On the GPU that would
// cost a cudaMalloc/cudaFree pair per call, so workspace here is cached per
// (device, stream) and only ever grows; the host-pointer entry points also
// keep per-thread device copies of A, B and C.
#include "runtime.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "internal.hpp"
#include "phase.hpp"

namespace mmsk {

// ------------------------------------------------------------------ errors
namespace {
thread_local std::string t_last_error;
}
void set_error_message(const std::string& msg) { t_last_error = msg; }
const char* last_error_message() { return t_last_error.c_str(); }

maxmulsk_status cuda_status(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return MAXMULSK_OK;
    set_error_message(std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    if (e == cudaErrorMemoryAllocation) return MAXMULSK_ERR_ALLOC;
    return MAXMULSK_ERR_CUDA;
}

// ------------------------------------------------------------------ devices
namespace {

struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct DeviceState {
    int sms = 0;
    int major = 0, minor = 0;
    int* err_word = nullptr;
    std::mutex mu;
    std::map<cudaStream_t, Workspace> ws;
};

std::mutex g_devices_mu;
std::vector<std::unique_ptr<DeviceState>> g_devices;

DeviceState* device_state(int dev) {
    std::lock_guard<std::mutex> lk(g_devices_mu);
    if ((int)g_devices.size() <= dev) g_devices.resize(dev + 1);
    if (!g_devices[dev]) {
        auto st = std::make_unique<DeviceState>();
        cudaDeviceGetAttribute(&st->sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&st->major, cudaDevAttrComputeCapabilityMajor, dev);
        cudaDeviceGetAttribute(&st->minor, cudaDevAttrComputeCapabilityMinor, dev);
        if (cudaMalloc(&st->err_word, sizeof(int)) == cudaSuccess) cudaMemset(st->err_word, 0, sizeof(int));
        else st->err_word = nullptr;
        g_devices[dev] = std::move(st);
    }
    return g_devices[dev].get();
}

DeviceState* current_state() {
    int dev = 0;
    cudaGetDevice(&dev);
    return device_state(dev);
}

// Per-thread device copies for the host-pointer entry points, and the
// streams and events of the row-block pipeline.
constexpr int kPipeBlocks = 8;
struct HostStage {
    cudaStream_t stream = nullptr;           // GEMM
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t b_in = nullptr;
    cudaEvent_t a_in[kPipeBlocks] = {};
    cudaEvent_t c_done[kPipeBlocks] = {};
    float* dA = nullptr; size_t capA = 0;
    float* dB = nullptr; size_t capB = 0;
    float* dC = nullptr; size_t capC = 0;
    float* dBp = nullptr; size_t capBp = 0;  // B's split planes (as floats)
};
thread_local std::map<int, HostStage> t_stage;

cudaError_t grow(float** p, size_t* cap, size_t need_elems) {
    if (*cap >= need_elems) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr; *cap = 0;
    cudaError_t e = cudaMalloc(p, need_elems * sizeof(float));
    if (e == cudaSuccess) *cap = need_elems;
    return e;
}

}  // namespace

int device_sm_count() { return current_state()->sms; }
int* device_error_word() { return current_state()->err_word; }

// ------------------------------------------------------------------ dispatch
bool handle_empty_dev(float* dC, size_t M, size_t K, size_t N, cudaStream_t s, maxmulsk_status* st) {
    if (M == 0 || N == 0) { *st = MAXMULSK_OK; return true; }
    if (K == 0) {
        *st = cuda_status(cudaMemsetAsync(dC, 0, M * N * sizeof(float), s), "cudaMemsetAsync(C)");
        return true;
    }
    return false;
}

maxmulsk_status run_plan_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                             const maxmulsk_plan& plan, void* ws, size_t ws_bytes, cudaStream_t s,
                             void* b_planes) {
    maxmulsk_status st = classify_plan(M, K, N, &plan);
    if (st != MAXMULSK_OK) return st;
    if (handle_empty_dev(dC, M, K, N, s, &st)) return st;
    if (!dA || !dB || !dC) { set_error_message("null matrix pointer"); return MAXMULSK_ERR_INVALID; }
    const size_t need = workspace_bytes(M, K, N, plan);
    if (need > 0 && (!ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(ws) & 255) != 0)) {
        set_error_message("workspace missing, too small or not 256-byte aligned");
        return MAXMULSK_ERR_INVALID;
    }
    DeviceState* ds = current_state();
    if (!ds->err_word) { set_error_message("device error word unavailable"); return MAXMULSK_ERR_ALLOC; }

    if (plan.precision == MAXMULSK_PREC_FP32) return simt_run(dA, dB, dC, M, K, N, plan, ws, ws_bytes, s);

    if (ds->major != 10) {
        set_error_message("split-precision tensor-core kernels need an sm_100 device");
        return MAXMULSK_ERR_UNSUPPORTED;
    }
    TcArgs a{};
    a.A = dA; a.B = dB; a.C = dC;
    a.M = (int64_t)M; a.K = (int64_t)K; a.N = (int64_t)N;
    a.precision = plan.precision;
    a.tile_m = plan.tile_m;
    a.tile_n = plan.tile_n;
    a.reuse_planes = (plan.variant == MAXMULSK_TC_REUSE_PLANES);
    // The fused split loads A and B with TMA: 16-byte aligned starts (row
    // lengths are checked by classify_plan). Otherwise the split-inputs path,
    // whose result is the same.
    a.fused = plan.variant == MAXMULSK_TC_FUSED_SPLIT && (reinterpret_cast<uintptr_t>(dA) & 15) == 0 &&
              (reinterpret_cast<uintptr_t>(dB) & 15) == 0 && b_planes == nullptr;
    a.split_k = plan.split_k;
    a.chunk = plan.chunk;
    a.err = ds->err_word;
    a.b_planes = a.reuse_planes ? nullptr : b_planes;
    if (!tc_bind_workspace(a, ws, ws_bytes)) {
        set_error_message("workspace too small for the tensor-core plan");
        return MAXMULSK_ERR_INVALID;
    }
    if (a.counters) {
        const size_t cb = tc_counter_bytes((int64_t)M, (int64_t)K, (int64_t)N, plan.precision, plan.tile_m,
                                         plan.tile_n, plan.split_k);
        if (cb > 0) {
            st = cuda_status(cudaMemsetAsync(a.counters, 0, cb, s), "cudaMemsetAsync(counters)");
            if (st != MAXMULSK_OK) return st;
        }
    }
    return cuda_status(tc_launch(a, s), "sgemm_split_tc launch");
}

void* managed_workspace(cudaStream_t s, size_t need, size_t* bytes, maxmulsk_status* st) {
    *st = MAXMULSK_OK;
    DeviceState* ds = current_state();
    std::lock_guard<std::mutex> lk(ds->mu);
    Workspace& w = ds->ws[s];
    if (w.bytes < need) {
        // The old buffer may still be read by work queued on this stream.
        if (w.ptr) {
            *st = cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            if (*st != MAXMULSK_OK) return nullptr;
            cudaFree(w.ptr);
            w.ptr = nullptr;
            w.bytes = 0;
        }
        size_t grown = need + need / 4;
        cudaError_t e = cudaMalloc(&w.ptr, grown);
        if (e != cudaSuccess) {
            w.ptr = nullptr;
            *st = cuda_status(e, "cudaMalloc(workspace)");
            return nullptr;
        }
        w.bytes = grown;
    }
    *bytes = w.bytes;
    return w.ptr;
}

maxmulsk_status run_plan_managed(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                 const maxmulsk_plan& plan, cudaStream_t s, void* b_planes) {
    maxmulsk_status st = classify_plan(M, K, N, &plan);
    if (st != MAXMULSK_OK) return st;
    if (handle_empty_dev(dC, M, K, N, s, &st)) return st;
    const size_t need = workspace_bytes(M, K, N, plan);
    void* ws = nullptr;
    size_t ws_bytes = 0;
    if (need > 0) {
        ws = managed_workspace(s, need, &ws_bytes, &st);
        if (!ws) return st;
    }
    return run_plan_dev(dA, dB, dC, M, K, N, plan, ws, ws_bytes, s, b_planes);
}

maxmulsk_status stream_status(cudaStream_t s) {
    maxmulsk_status st = cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (st != MAXMULSK_OK) return st;
    DeviceState* ds = current_state();
    if (!ds->err_word) return MAXMULSK_OK;
    int flag = 0;
    st = cuda_status(cudaMemcpy(&flag, ds->err_word, sizeof(int), cudaMemcpyDeviceToHost), "read error word");
    if (st != MAXMULSK_OK) return st;
    if (flag != 0) {
        cudaMemset(ds->err_word, 0, sizeof(int));
        set_error_message("a bounded device-side wait timed out");
        return MAXMULSK_ERR_TIMEOUT;
    }
    return MAXMULSK_OK;
}

namespace {

bool page_locked(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

maxmulsk_status ensure_pipeline(HostStage& hs) {
    maxmulsk_status st = MAXMULSK_OK;
    if (!hs.h2d) st = cuda_status(cudaStreamCreateWithFlags(&hs.h2d, cudaStreamNonBlocking), "cudaStreamCreate");
    if (st == MAXMULSK_OK && !hs.d2h)
        st = cuda_status(cudaStreamCreateWithFlags(&hs.d2h, cudaStreamNonBlocking), "cudaStreamCreate");
    if (st == MAXMULSK_OK && !hs.b_in) st = cuda_status(cudaEventCreateWithFlags(&hs.b_in, cudaEventDisableTiming), "cudaEventCreate");
    for (int i = 0; i < kPipeBlocks && st == MAXMULSK_OK; i++) {
        if (!hs.a_in[i]) st = cuda_status(cudaEventCreateWithFlags(&hs.a_in[i], cudaEventDisableTiming), "cudaEventCreate");
        if (st == MAXMULSK_OK && !hs.c_done[i])
            st = cuda_status(cudaEventCreateWithFlags(&hs.c_done[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    return st;
}

// Row-block pipeline. B is copied first; A is copied in kPipeBlocks row
// blocks on one copy stream, each block's GEMM starts when its rows have
// arrived, and each block of C goes back on a second copy stream as soon as
// it is written. The PCIe link carries A in one direction while it carries C
// in the other, so the call costs about copy(B) + copy(A) + one block,
// instead of copy(A, B) + GEMM + copy(C). Each row of C is the same
// computation as in a whole-matrix launch of the same plan (the K slicing
// does not depend on M); only the tensor-core schedule's tail-wave K split,
// which depends on the tile count, can differ.
maxmulsk_status host_pipelined(HostStage& hs, const float* A, const float* B, float* C, size_t M, size_t K,
                               size_t N, const maxmulsk_plan& plan) {
    maxmulsk_status st = ensure_pipeline(hs);
    if (st != MAXMULSK_OK) return st;
    size_t rows = (M + kPipeBlocks - 1) / kPipeBlocks;
    rows = (rows + 255) / 256 * 256;
    const int nblk = (int)((M + rows - 1) / rows);
    cudaStream_t s = hs.stream;
    auto fail = [&](maxmulsk_status e) {
        cudaStreamSynchronize(hs.h2d);
        cudaStreamSynchronize(s);
        cudaStreamSynchronize(hs.d2h);
        return e;
    };

    {
        PhaseScope ps(kPhaseH2D, hs.h2d);
        st = cuda_status(cudaMemcpyAsync(hs.dB, B, K * N * sizeof(float), cudaMemcpyHostToDevice, hs.h2d), "copy B");
    }
    if (st != MAXMULSK_OK) return fail(st);
    st = cuda_status(cudaEventRecord(hs.b_in, hs.h2d), "cudaEventRecord");
    if (st != MAXMULSK_OK) return fail(st);
    for (int i = 0; i < nblk; i++) {
        const size_t r0 = (size_t)i * rows, mb = std::min(rows, M - r0);
        {
            PhaseScope ps(kPhaseH2D, hs.h2d);
            st = cuda_status(cudaMemcpyAsync(hs.dA + r0 * K, A + r0 * K, mb * K * sizeof(float),
                                             cudaMemcpyHostToDevice, hs.h2d), "copy A block");
        }
        if (st != MAXMULSK_OK) return fail(st);
        st = cuda_status(cudaEventRecord(hs.a_in[i], hs.h2d), "cudaEventRecord");
        if (st != MAXMULSK_OK) return fail(st);
    }

    st = cuda_status(cudaStreamWaitEvent(s, hs.b_in, 0), "cudaStreamWaitEvent");
    if (st != MAXMULSK_OK) return fail(st);
    void* b_planes = nullptr;
    if (plan.precision != MAXMULSK_PREC_FP32 && plan.variant != MAXMULSK_TC_FUSED_SPLIT) {
        // B's planes once for all blocks (the fused split makes none).
        const size_t nb = split_one_bytes((int64_t)K, (int64_t)N, plan.precision, true);
        st = cuda_status(grow(&hs.dBp, &hs.capBp, (nb + sizeof(float) - 1) / sizeof(float)), "cudaMalloc(B planes)");
        if (st != MAXMULSK_OK) return fail(st);
        {
            PhaseScope ps(kPhaseSplit, s);
            st = cuda_status(split_one(hs.dB, (int64_t)K, (int64_t)N, plan.precision, true, hs.dBp, s), "split B");
        }
        if (st != MAXMULSK_OK) return fail(st);
        b_planes = hs.dBp;
    }
    for (int i = 0; i < nblk; i++) {
        const size_t r0 = (size_t)i * rows, mb = std::min(rows, M - r0);
        st = cuda_status(cudaStreamWaitEvent(s, hs.a_in[i], 0), "cudaStreamWaitEvent");
        if (st != MAXMULSK_OK) return fail(st);
        st = run_plan_managed(hs.dA + r0 * K, hs.dB, hs.dC + r0 * N, mb, K, N, plan, s, b_planes);
        if (st != MAXMULSK_OK) return fail(st);
        st = cuda_status(cudaEventRecord(hs.c_done[i], s), "cudaEventRecord");
        if (st != MAXMULSK_OK) return fail(st);
        st = cuda_status(cudaStreamWaitEvent(hs.d2h, hs.c_done[i], 0), "cudaStreamWaitEvent");
        if (st != MAXMULSK_OK) return fail(st);
        {
            PhaseScope ps(kPhaseD2H, hs.d2h);
            st = cuda_status(cudaMemcpyAsync(C + r0 * N, hs.dC + r0 * N, mb * N * sizeof(float),
                                             cudaMemcpyDeviceToHost, hs.d2h), "copy C block");
        }
        if (st != MAXMULSK_OK) return fail(st);
    }
    st = cuda_status(cudaStreamSynchronize(hs.d2h), "cudaStreamSynchronize");
    if (st != MAXMULSK_OK) return fail(st);
    return stream_status(s);
}

}  // namespace

void autotune_fallback_host(const float* A, const float* B, size_t M, size_t K, size_t N, int precision) {
    if (M == 0 || N == 0 || K == 0 || !A || !B) return;
    if (!autotune_fallback_enabled() || !picker_doubt(M, K, N, precision)) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    HostStage& hs = t_stage[dev];
    if (!hs.stream && cudaStreamCreateWithFlags(&hs.stream, cudaStreamNonBlocking) != cudaSuccess) {
        hs.stream = nullptr;
        return;
    }
    if (grow(&hs.dA, &hs.capA, M * K) != cudaSuccess || grow(&hs.dB, &hs.capB, K * N) != cudaSuccess ||
        grow(&hs.dC, &hs.capC, M * N) != cudaSuccess)
        return;
    cudaStream_t s = hs.stream;
    if (cudaMemcpyAsync(hs.dA, A, M * K * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(hs.dB, B, K * N * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess) {
        cudaStreamSynchronize(s);
        return;
    }
    autotune_fallback(hs.dA, hs.dB, hs.dC, M, K, N, precision, s);
}

maxmulsk_status run_plan_host(const float* A, const float* B, float* C, size_t M, size_t K, size_t N,
                              const maxmulsk_plan& plan) {
    maxmulsk_status st = classify_plan(M, K, N, &plan);
    if (st != MAXMULSK_OK) return st;
    if (M == 0 || N == 0) return MAXMULSK_OK;
    if (!C) { set_error_message("null C"); return MAXMULSK_ERR_INVALID; }
    if (K == 0) { std::memset(C, 0, M * N * sizeof(float)); return MAXMULSK_OK; }
    if (!A || !B) { set_error_message("null A or B"); return MAXMULSK_ERR_INVALID; }

    int dev = 0;
    st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != MAXMULSK_OK) return st;
    HostStage& hs = t_stage[dev];
    if (!hs.stream) {
        st = cuda_status(cudaStreamCreateWithFlags(&hs.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        if (st != MAXMULSK_OK) return st;
    }
    if ((st = cuda_status(grow(&hs.dA, &hs.capA, M * K), "cudaMalloc(A)")) != MAXMULSK_OK) return st;
    if ((st = cuda_status(grow(&hs.dB, &hs.capB, K * N), "cudaMalloc(B)")) != MAXMULSK_OK) return st;
    if ((st = cuda_status(grow(&hs.dC, &hs.capC, M * N), "cudaMalloc(C)")) != MAXMULSK_OK) return st;

    // The pipeline pays off once the copies dominate; it needs page-locked A
    // and C, since copies from pageable memory do not overlap with anything.
    const size_t streamed = (M * K + M * N) * sizeof(float);
    const bool planes_given = plan.precision != MAXMULSK_PREC_FP32 && plan.variant == MAXMULSK_TC_REUSE_PLANES;
    if (M >= 1024 && streamed >= (32u << 20) && !planes_given && page_locked(A) && page_locked(C))
        return host_pipelined(hs, A, B, C, M, K, N, plan);

    cudaStream_t s = hs.stream;
    {
        PhaseScope ps(kPhaseH2D, s);
        st = cuda_status(cudaMemcpyAsync(hs.dA, A, M * K * sizeof(float), cudaMemcpyHostToDevice, s), "copy A");
        if (st == MAXMULSK_OK)
            st = cuda_status(cudaMemcpyAsync(hs.dB, B, K * N * sizeof(float), cudaMemcpyHostToDevice, s), "copy B");
    }
    if (st != MAXMULSK_OK) return st;
    st = run_plan_managed(hs.dA, hs.dB, hs.dC, M, K, N, plan, s);
    if (st != MAXMULSK_OK) { cudaStreamSynchronize(s); return st; }
    {
        PhaseScope ps(kPhaseD2H, s);
        st = cuda_status(cudaMemcpyAsync(C, hs.dC, M * N * sizeof(float), cudaMemcpyDeviceToHost, s), "copy C");
    }
    if (st != MAXMULSK_OK) { cudaStreamSynchronize(s); return st; }
    return stream_status(s);
}

}  // namespace mmsk
