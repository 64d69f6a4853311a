// Phase timing (phase.hpp): CUDA event pairs per phase scope, summed per
// phase on request; NVTX ranges on the host.
#include "phase.hpp"

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "maxmulsk.h"

namespace mmsk {
namespace {

const char* const kPhaseNames[kPhaseCount] = {"split", "gemm", "reduce", "grouped", "h2d", "d2h"};

std::atomic<int> g_on{-1};               // -1: MAXMULSK_PHASE_TIMING not read yet

struct Record {
    int phase;
    int device;
    cudaEvent_t begin, end;
};

std::mutex g_mu;
std::vector<Record> g_records;           // recorded since the last report
constexpr size_t kMaxRecords = 1 << 16;  // beyond this, scopes record nothing until the next report

thread_local int t_muted = 0;             // PhaseMute nesting depth on this thread

}  // namespace

PhaseMute::PhaseMute() { t_muted++; }
PhaseMute::~PhaseMute() { t_muted--; }

bool phase_timing_on() {
    int v = g_on.load(std::memory_order_relaxed);
    if (v >= 0) return v == 1;
    const char* e = std::getenv("MAXMULSK_PHASE_TIMING");
    const int env = (e && *e && std::strcmp(e, "0") != 0) ? 1 : 0;
    int expected = -1;
    g_on.compare_exchange_strong(expected, env);
    return g_on.load(std::memory_order_relaxed) == 1;
}

void phase_set(bool on) { g_on.store(on ? 1 : 0); }

PhaseScope::PhaseScope(Phase phase, cudaStream_t stream) : phase_(phase), stream_(stream) {
    if (t_muted > 0 || !phase_timing_on()) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    if (cudaEventCreate(&begin_) != cudaSuccess) { begin_ = nullptr; return; }
    if (cudaEventRecord(begin_, stream) != cudaSuccess) {
        cudaEventDestroy(begin_);
        begin_ = nullptr;
        return;
    }
    nvtxRangePushA(kPhaseNames[phase]);
    nvtx_ = true;
}

PhaseScope::~PhaseScope() {
    if (nvtx_) nvtxRangePop();
    if (!begin_) return;
    cudaEvent_t end = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaEventCreate(&end) != cudaSuccess || cudaEventRecord(end, stream_) != cudaSuccess) {
        if (end) cudaEventDestroy(end);
        cudaEventDestroy(begin_);
        return;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_records.size() >= kMaxRecords) {
        cudaEventDestroy(begin_);
        cudaEventDestroy(end);
        return;
    }
    g_records.push_back(Record{phase_, dev, begin_, end});
}

size_t phase_report(char* buf, size_t len) {
    std::vector<Record> recs;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        recs.swap(g_records);
    }
    double ms[kPhaseCount] = {};
    long calls[kPhaseCount] = {};
    int cur = -1;
    if (!recs.empty()) cudaGetDevice(&cur);
    for (const Record& r : recs) {
        cudaSetDevice(r.device);
        float t = 0.f;
        if (cudaEventSynchronize(r.end) == cudaSuccess && cudaEventElapsedTime(&t, r.begin, r.end) == cudaSuccess) {
            ms[r.phase] += t;
            calls[r.phase]++;
        }
        cudaEventDestroy(r.begin);
        cudaEventDestroy(r.end);
    }
    if (cur >= 0) cudaSetDevice(cur);
    std::string out = "{";
    for (int p = 0; p < kPhaseCount; p++) {
        if (!calls[p]) continue;
        char item[128];
        std::snprintf(item, sizeof item, "%s\"%s\": {\"calls\": %ld, \"ms\": %.9g}", out.size() > 1 ? ", " : "",
                      kPhaseNames[p], calls[p], ms[p]);
        out += item;
    }
    out += "}";
    if (buf && len) {
        const size_t n = out.size() < len - 1 ? out.size() : len - 1;
        std::memcpy(buf, out.data(), n);
        buf[n] = '\0';
    }
    return out.size();
}

}  // namespace mmsk
