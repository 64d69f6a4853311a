// Grouped launches: many independent GEMMs of uneven shapes in one persistent
// kernel, captured once into a CUDA graph and replayed.
//
// The reference's counterpart is run_batch (sme/v3/sme-1x4-acc-kcout-onestream.hpp:61-63,
// .cpp:598-605): one streaming region for a list of Gemm{A, B, C, M, K, N},
// blocking chosen per GEMM. Here the list becomes a table in device memory,
// every GEMM is cut into (tile, K slice) units, the units are sorted heaviest
// first, and one persistent kernel takes them from an atomic counter
// (simt.cu, sgemm_simt_grouped_kernel). The tile shape is one per group; the
// K split is chosen per problem so that no unit is much longer than the
// average share of an SM.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "internal.hpp"
#include "runtime.hpp"

struct maxmulsk_grouped_s {
    int device = 0;
    maxmulsk_plan plan{};
    size_t count = 0;
    std::vector<int32_t> split_k;          // per problem, as planned
    mmsk::GroupProblem* d_probs = nullptr;
    mmsk::GroupUnit* d_units = nullptr;
    int nunits = 0;
    unsigned* d_next = nullptr;
    void* d_scratch = nullptr;             // [counters of all split problems][partials]
    size_t counter_bytes = 0;
    int grid = 0;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace mmsk {
namespace {

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Relative throughput of the SIMT tile shapes (measured at 4096^3: 48, 41 and
// 32 TFLOP/s for 128x128, 128x64, 64x64).
double tile_rate(int bm, int bn) {
    if (bm == 128 && bn == 128) return 1.0;
    if (bm == 128 && bn == 64) return 0.85;
    return 0.66;
}

// Padded work of a problem on a tile shape, in multiply-adds.
double padded_work(const maxmulsk_problem& p, int bm, int bn) {
    return (double)((p.M + bm - 1) / bm * bm) * (double)((p.N + bn - 1) / bn * bn) * (double)p.K;
}

// The tile shape with the least estimated time for the whole group.
void pick_tile(const maxmulsk_problem* probs, size_t n, int* bm, int* bn) {
    const int cands[3][2] = {{128, 128}, {128, 64}, {64, 64}};
    double best = -1;
    for (auto& c : cands) {
        double t = 0;
        for (size_t i = 0; i < n; i++) t += padded_work(probs[i], c[0], c[1]);
        t /= tile_rate(c[0], c[1]);
        if (best < 0 || t < best) { best = t; *bm = c[0]; *bn = c[1]; }
    }
}

}  // namespace
}  // namespace mmsk

using namespace mmsk;

extern "C" {

maxmulsk_status maxmulsk_grouped_create(const maxmulsk_problem* problems, size_t count, const maxmulsk_plan* group_plan,
                                        maxmulsk_grouped* out) {
    if (!out) return MAXMULSK_ERR_INVALID;
    *out = nullptr;
    if (count > 0 && !problems) { set_error_message("null problem list"); return MAXMULSK_ERR_INVALID; }
    for (size_t i = 0; i < count; i++) {
        const maxmulsk_problem& p = problems[i];
        if (p.M && p.N && (!p.C || (p.K && (!p.A || !p.B)))) {
            set_error_message("null matrix pointer in a grouped problem");
            return MAXMULSK_ERR_INVALID;
        }
        if (p.M > 0x7FFFFFFFull || p.N > 0x7FFFFFFFull || p.K > 0x7FFFFFFFull || (p.M + 63) / 64 > 65535) {
            set_error_message("grouped problem too large");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
    }
    maxmulsk_plan plan;
    std::memset(&plan, 0, sizeof plan);
    plan.precision = MAXMULSK_PREC_FP32;
    if (group_plan) {
        plan = *group_plan;
        maxmulsk_plan probe = plan;
        if (probe.split_k == 0) probe.split_k = 1;            // 0 = per problem, picked here
        maxmulsk_status st = classify_plan(1, 1, 1, &probe);
        if (st != MAXMULSK_OK) return st;
        if (plan.precision != MAXMULSK_PREC_FP32) {
            set_error_message("grouped launches run FP32 plans");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
    } else {
        pick_tile(problems, count, &plan.tile_m, &plan.tile_n);
        plan.split_k = 0;
    }
    const int bm = plan.tile_m, bn = plan.tile_n;

    std::unique_ptr<maxmulsk_grouped_s> g(new (std::nothrow) maxmulsk_grouped_s());
    if (!g) return MAXMULSK_ERR_ALLOC;
    cudaGetDevice(&g->device);
    g->plan = plan;
    g->count = count;
    g->split_k.assign(count, 1);
    const int sms = device_sm_count() > 0 ? device_sm_count() : 148;

    // Per-problem K split: units no longer than a quarter of an SM's average
    // share of the group, slices at least 256 deep.
    double total = 0;
    for (size_t i = 0; i < count; i++) total += padded_work(problems[i], bm, bn);
    const double cap = std::max(1.0, total / (4.0 * 2.0 * sms));      // 2 CTAs per SM
    for (size_t i = 0; i < count; i++) {
        const maxmulsk_problem& p = problems[i];
        if (!p.M || !p.N || !p.K) continue;
        int s = 1;
        if (plan.split_k > 0) {
            s = plan.split_k;
        } else {
            const double unit = (double)bm * bn * (double)p.K;
            s = (int)std::min<double>(64.0, std::ceil(unit / cap));
            const int kmax = (int)std::max<size_t>(1, p.K / 256);
            s = std::max(1, std::min(s, kmax));
        }
        g->split_k[i] = slice_count(p.K, s) > 1 ? s : 1;
    }

    // Tables, scratch layout and units.
    std::vector<GroupProblem> hp(count);
    std::vector<GroupUnit> hu;
    size_t counters = 0, partials = 0;
    std::vector<size_t> ctr_off(count, 0), part_off(count, 0);
    for (size_t i = 0; i < count; i++) {
        const maxmulsk_problem& p = problems[i];
        const int splits = (p.K ? slice_count(p.K, g->split_k[i]) : 1);
        const size_t tiles = (size_t)((p.M + bm - 1) / bm) * ((p.N + bn - 1) / bn);
        if (splits > 1) {
            ctr_off[i] = counters;
            counters += tiles * sizeof(unsigned);
            part_off[i] = partials;
            partials += align256((size_t)splits * p.M * p.N * sizeof(float));
        }
    }
    g->counter_bytes = align256(counters);
    const size_t scratch_bytes = g->counter_bytes + partials;
    if (scratch_bytes) {
        cudaError_t e = cudaMalloc(&g->d_scratch, scratch_bytes);
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(grouped scratch)");
    }
    for (size_t i = 0; i < count; i++) {
        const maxmulsk_problem& p = problems[i];
        GroupProblem& q = hp[i];
        std::memset(&q, 0, sizeof q);
        q.a.A = p.A; q.a.B = p.B; q.a.C = p.C;
        q.a.M = (int64_t)p.M; q.a.K = (int64_t)p.K; q.a.N = (int64_t)p.N;
        q.a.kchunk = (int64_t)slice_len(p.K, g->split_k[i]);
        q.a.splits = p.K ? slice_count(p.K, g->split_k[i]) : 1;
        q.tiles_n = (int32_t)((p.N + bn - 1) / bn);
        q.vec = (p.K % 4 == 0) && (p.N % 4 == 0) && ((uintptr_t)p.A % 16 == 0) && ((uintptr_t)p.B % 16 == 0) &&
                ((uintptr_t)p.C % 16 == 0);
        if (q.a.splits > 1) {
            q.a.counters = reinterpret_cast<unsigned*>(static_cast<char*>(g->d_scratch) + ctr_off[i]);
            q.a.partial = reinterpret_cast<float*>(static_cast<char*>(g->d_scratch) + g->counter_bytes + part_off[i]);
        }
        if (!p.M || !p.N || !p.K) continue;                   // handled by memsets below
        const int tm_n = (int)((p.M + bm - 1) / bm), tn_n = q.tiles_n;
        for (int z = 0; z < q.a.splits; z++)
            for (int tm = 0; tm < tm_n; tm++)
                for (int tn = 0; tn < tn_n; tn++) hu.push_back(GroupUnit{(int32_t)i, tm, tn, z});
    }
    // Heaviest units first (K slice length), stable so slices stay grouped.
    std::stable_sort(hu.begin(), hu.end(), [&](const GroupUnit& x, const GroupUnit& y) {
        const GroupProblem& a = hp[x.problem];
        const GroupProblem& b = hp[y.problem];
        const int64_t la = std::min(a.a.kchunk, a.a.K - (int64_t)x.z * a.a.kchunk);
        const int64_t lb = std::min(b.a.kchunk, b.a.K - (int64_t)y.z * b.a.kchunk);
        return la > lb;
    });
    g->nunits = (int)hu.size();
    g->grid = std::max(1, std::min(g->nunits, 2 * sms));

    cudaError_t e;
    if ((e = cudaMalloc(&g->d_probs, std::max<size_t>(1, count) * sizeof(GroupProblem))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_units, std::max<size_t>(1, hu.size()) * sizeof(GroupUnit))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_next, sizeof(unsigned))) != cudaSuccess) {
        maxmulsk_grouped_destroy(g.release());
        return cuda_status(e, "cudaMalloc(grouped tables)");
    }
    if (count) cudaMemcpy(g->d_probs, hp.data(), count * sizeof(GroupProblem), cudaMemcpyHostToDevice);
    if (!hu.empty()) cudaMemcpy(g->d_units, hu.data(), hu.size() * sizeof(GroupUnit), cudaMemcpyHostToDevice);
    if (g->d_scratch && g->counter_bytes) cudaMemset(g->d_scratch, 0, g->counter_bytes);

    // Capture: K == 0 problems are zero-filled; the unit counter and the
    // split-K arrival counters are reset; then the one persistent kernel.
    e = cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) { maxmulsk_grouped_destroy(g.release()); return cuda_status(e, "cudaStreamCreate"); }
    e = cudaStreamBeginCapture(g->cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (size_t i = 0; i < count; i++)
            if (problems[i].M && problems[i].N && !problems[i].K)
                cudaMemsetAsync(problems[i].C, 0, problems[i].M * problems[i].N * sizeof(float), g->cap);
        cudaMemsetAsync(g->d_next, 0, sizeof(unsigned), g->cap);
        if (g->d_scratch && g->counter_bytes) cudaMemsetAsync(g->d_scratch, 0, g->counter_bytes, g->cap);
        if (g->nunits > 0)
            simt_grouped_launch(g->d_probs, g->d_units, g->nunits, g->d_next, bm, bn, plan.variant, g->grid, g->cap);
        cudaError_t e2 = cudaStreamEndCapture(g->cap, &g->graph);
        if (e == cudaSuccess) e = e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
        maxmulsk_grouped_destroy(g.release());
        return cuda_status(e, "grouped graph capture");
    }
    *out = g.release();
    return MAXMULSK_OK;
}

maxmulsk_status maxmulsk_grouped_launch(maxmulsk_grouped g, void* stream) {
    if (!g || !g->exec) return MAXMULSK_ERR_INVALID;
    return cuda_status(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch(grouped)");
}

maxmulsk_status maxmulsk_grouped_info(maxmulsk_grouped g, maxmulsk_plan* group_plan, int32_t* split_k,
                                      size_t* units) {
    if (!g) return MAXMULSK_ERR_INVALID;
    if (group_plan) *group_plan = g->plan;
    if (split_k) std::memcpy(split_k, g->split_k.data(), g->count * sizeof(int32_t));
    if (units) *units = (size_t)g->nunits;
    return MAXMULSK_OK;
}

void maxmulsk_grouped_destroy(maxmulsk_grouped g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->cap) { cudaStreamSynchronize(g->cap); cudaStreamDestroy(g->cap); }
    cudaFree(g->d_probs);
    cudaFree(g->d_units);
    cudaFree(g->d_next);
    cudaFree(g->d_scratch);
    delete g;
}

maxmulsk_status maxmulsk_sgemm_grouped_dev(const maxmulsk_problem* problems, size_t count, void* stream) {
    maxmulsk_grouped g = nullptr;
    maxmulsk_status st = maxmulsk_grouped_create(problems, count, nullptr, &g);
    if (st != MAXMULSK_OK) return st;
    st = maxmulsk_grouped_launch(g, stream);
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    maxmulsk_grouped_destroy(g);
    if (st != MAXMULSK_OK) return st;
    return cuda_status(e, "cudaStreamSynchronize(grouped)");
}

}  // extern "C"
