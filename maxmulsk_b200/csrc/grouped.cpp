// Grouped launches: many independent GEMMs of uneven shapes in one persistent
// kernel, captured once into a CUDA graph and replayed; how the group is cut
// into work is chosen by timing candidate graphs (an exhaustive search over a
// few group configurations) unless the caller fixes it.
//
// The reference's counterpart is run_batch (sme/v3/sme-1x4-acc-kcout-onestream.hpp:61-63,
// .cpp:598-605): one streaming region for a list of Gemm{A, B, C, M, K, N},
// blocking chosen per GEMM. Here the list becomes a table in device memory,
// every GEMM is cut into (tile, K slice) units, the units are sorted heaviest
// first, and one persistent kernel runs them:
//   * FP32 groups: sgemm_simt_grouped_kernel (simt.cu), units taken from an
//     atomic counter; one tile shape per group, the K split chosen per problem
//     so that no unit is much longer than the average share of an SM;
//   * split-precision groups (BF16x6 / BF16x9): the fused-split tcgen05 kernel
//     (tc.cu, tc_fused_kernel) over tables of problems, units and per-problem
//     FP32 tensor maps, 128 x 128 tiles. TMA needs rows that start on 16-byte
//     boundaries: an A whose K is not a multiple of 4 (or that is not 16-byte
//     aligned) is copied, inside the same graph, into a zero-padded buffer of
//     the group with rows of a multiple of 4 floats. A problem whose B cannot
//     be read that way (N not a multiple of 4, B not 16-byte aligned) runs in
//     the FP32 grouped kernel captured in the same graph, at FP32 accuracy;
//   * split-precision problems of at least `single_gflop` GFLOP whose own
//     picked plan (tuning database, learned model, rule) is not the fused
//     split run as their own launches of that plan (split pre-pass +
//     tcgen05 GEMM on larger tiles) in the same graph, after the persistent
//     kernel: a problem big enough to fill the GPU on its own gains more from
//     its best plan than from sharing the fused kernel's 128 x 128 tiles.
//
// Configuration search (maxmulsk_grouped_create with no K split given): each
// candidate -- FP32: tile shape x K-split policy; split precision: the fused
// part's K-split policy x the single-launch threshold -- is built, captured,
// replayed once to warm and three times timed (median), and the fastest is
// kept: the group-level counterpart of maxmulsk_autotune_dev. It runs the
// group, so C is written while the group is created.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "internal.hpp"
#include "phase.hpp"
#include "runtime.hpp"

struct maxmulsk_grouped_s {
    int device = 0;
    maxmulsk_plan plan{};
    size_t count = 0;
    std::vector<int32_t> split_k;          // per problem, as planned
    // FP32 part
    maxmulsk_plan simt_plan{};
    mmsk::GroupProblem* d_probs = nullptr;
    mmsk::GroupUnit* d_units = nullptr;
    int nunits = 0;
    unsigned* d_next = nullptr;
    void* d_scratch = nullptr;             // [counters of all split problems][partials]
    size_t counter_bytes = 0;
    int grid = 0;
    // split-precision part
    void* d_tc = nullptr;                  // [problems][units][tensor maps][counters][partials]
    mmsk::TcGroupArgs tc{};
    size_t tc_counter_bytes = 0;
    void* tc_counters = nullptr;
    int tc_grid = 0;
    struct Repack {                        // A copied to a 16-byte pitch before each launch
        float* dst;
        const float* src;
        size_t rows, cols, dst_ld;
    };
    std::vector<Repack> repack;
    void* d_apad = nullptr;
    // split-precision problems run as their own launches
    struct Single {
        size_t problem;
        maxmulsk_plan plan;
    };
    std::vector<Single> singles;
    void* d_single_ws = nullptr;           // shared by the singles (one after another on one stream)
    size_t single_ws_bytes = 0;
    std::vector<maxmulsk_plan> plans;      // per problem, as run
    // the captured graph
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

bool runs(const maxmulsk_problem& p) { return p.M && p.N && p.K; }

// The tile shape with the least estimated time for the problems `idx`.
void pick_tile(const maxmulsk_problem* probs, const std::vector<size_t>& idx, int* bm, int* bn) {
    const int cands[3][2] = {{128, 128}, {128, 64}, {64, 64}};
    double best = -1;
    for (auto& c : cands) {
        double t = 0;
        for (size_t i : idx) t += padded_work(probs[i], c[0], c[1]);
        t /= tile_rate(c[0], c[1]);
        if (best < 0 || t < best) { best = t; *bm = c[0]; *bn = c[1]; }
    }
}

// K split of each problem: units no longer than 1/share of a work slot's
// average share of the group, slices at least 256 deep, at most 64 slices.
// fixed > 0 imposes that split on every problem; share <= 0 splits none.
std::vector<int> plan_splits(const maxmulsk_problem* probs, const std::vector<size_t>& idx, int bm, int bn,
                             int slots, int fixed, double share) {
    double total = 0;
    for (size_t i : idx) total += padded_work(probs[i], bm, bn);
    if (fixed <= 0 && share <= 0) return std::vector<int>(idx.size(), 1);
    const double cap = std::max(1.0, total / (share * slots));
    std::vector<int> out(idx.size(), 1);
    for (size_t j = 0; j < idx.size(); j++) {
        const maxmulsk_problem& p = probs[idx[j]];
        if (!runs(p)) continue;
        int s = 1;
        if (fixed > 0) {
            s = fixed;
        } else {
            const double unit = (double)bm * bn * (double)p.K;
            s = (int)std::min<double>(64.0, std::ceil(unit / cap));
            const int kmax = (int)std::max<size_t>(1, p.K / 256);
            s = std::max(1, std::min(s, kmax));
        }
        out[j] = slice_count(p.K, s) > 1 ? s : 1;
    }
    return out;
}

// FP32 part: the problems `idx` on the SIMT grouped kernel.
maxmulsk_status build_simt(maxmulsk_grouped_s* g, const maxmulsk_problem* problems, const std::vector<size_t>& idx,
                           const maxmulsk_plan& plan, double share, int sms) {
    const int bm = plan.tile_m, bn = plan.tile_n;
    const std::vector<int> sk = plan_splits(problems, idx, bm, bn, 2 * sms, plan.split_k, share);   // 2 CTAs per SM
    for (size_t j = 0; j < idx.size(); j++) {
        g->split_k[idx[j]] = sk[j];
        maxmulsk_plan& q = g->plans[idx[j]];
        q = plan;
        q.split_k = sk[j];
    }

    std::vector<GroupProblem> hp(idx.size());
    std::vector<GroupUnit> hu;
    size_t counters = 0, partials = 0;
    std::vector<size_t> ctr_off(idx.size(), 0), part_off(idx.size(), 0);
    for (size_t j = 0; j < idx.size(); j++) {
        const maxmulsk_problem& p = problems[idx[j]];
        const int splits = (p.K ? slice_count(p.K, sk[j]) : 1);
        const size_t tiles = (size_t)((p.M + bm - 1) / bm) * ((p.N + bn - 1) / bn);
        if (splits > 1) {
            ctr_off[j] = counters;
            counters += tiles * sizeof(unsigned);
            part_off[j] = partials;
            partials += align256((size_t)splits * p.M * p.N * sizeof(float));
        }
    }
    g->counter_bytes = align256(counters);
    const size_t scratch_bytes = g->counter_bytes + partials;
    if (scratch_bytes) {
        cudaError_t e = cudaMalloc(&g->d_scratch, scratch_bytes);
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(grouped scratch)");
    }
    for (size_t j = 0; j < idx.size(); j++) {
        const maxmulsk_problem& p = problems[idx[j]];
        GroupProblem& q = hp[j];
        std::memset(&q, 0, sizeof q);
        q.a.A = p.A; q.a.B = p.B; q.a.C = p.C;
        q.a.M = (int64_t)p.M; q.a.K = (int64_t)p.K; q.a.N = (int64_t)p.N;
        q.a.kchunk = (int64_t)slice_len(p.K, sk[j]);
        q.a.splits = p.K ? slice_count(p.K, sk[j]) : 1;
        q.tiles_n = (int32_t)((p.N + bn - 1) / bn);
        q.vec = (p.K % 4 == 0) && (p.N % 4 == 0) && ((uintptr_t)p.A % 16 == 0) && ((uintptr_t)p.B % 16 == 0) &&
                ((uintptr_t)p.C % 16 == 0);
        if (q.a.splits > 1) {
            q.a.counters = reinterpret_cast<unsigned*>(static_cast<char*>(g->d_scratch) + ctr_off[j]);
            q.a.partial = reinterpret_cast<float*>(static_cast<char*>(g->d_scratch) + g->counter_bytes + part_off[j]);
        }
        if (!runs(p)) continue;                               // handled by memsets
        const int tm_n = (int)((p.M + bm - 1) / bm), tn_n = q.tiles_n;
        for (int z = 0; z < q.a.splits; z++)
            for (int tm = 0; tm < tm_n; tm++)
                for (int tn = 0; tn < tn_n; tn++) hu.push_back(GroupUnit{(int32_t)j, tm, tn, z});
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
    if ((e = cudaMalloc(&g->d_probs, std::max<size_t>(1, idx.size()) * sizeof(GroupProblem))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_units, std::max<size_t>(1, hu.size()) * sizeof(GroupUnit))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_next, sizeof(unsigned))) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(grouped tables)");
    if (!idx.empty() && (e = cudaMemcpy(g->d_probs, hp.data(), idx.size() * sizeof(GroupProblem),
                                        cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_status(e, "upload grouped problems");
    if (!hu.empty() && (e = cudaMemcpy(g->d_units, hu.data(), hu.size() * sizeof(GroupUnit),
                                       cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_status(e, "upload grouped units");
    if (g->d_scratch && g->counter_bytes) cudaMemset(g->d_scratch, 0, g->counter_bytes);
    return MAXMULSK_OK;
}

// Split-precision part: the problems `idx` on the fused-split tcgen05 kernel.
maxmulsk_status build_tc(maxmulsk_grouped_s* g, const maxmulsk_problem* problems, const std::vector<size_t>& idx,
                         int precision, int fixed_split, double share, int sms) {
    constexpr int T = 128;                                    // tile rows and columns
    const std::vector<int> sk = plan_splits(problems, idx, T, T, sms, fixed_split, share);   // 1 CTA per SM
    const size_t n = idx.size();
    for (size_t j = 0; j < n; j++) {
        maxmulsk_plan& q = g->plans[idx[j]];
        std::memset(&q, 0, sizeof q);
        q.precision = precision; q.tile_m = T; q.tile_n = T; q.split_k = sk[j]; q.variant = MAXMULSK_TC_FUSED_SPLIT;
    }
    std::vector<TcGroupProblem> hp(n);
    std::vector<TcGroupUnit> hu;
    std::vector<unsigned char> maps(256 * std::max<size_t>(1, n));
    size_t counters = 0, partials = 0;
    std::vector<size_t> ctr_off(n, 0), part_off(n, 0);
    for (size_t j = 0; j < n; j++) {
        const maxmulsk_problem& p = problems[idx[j]];
        g->split_k[idx[j]] = sk[j];
        const int splits = slice_count(p.K, sk[j]);
        const int64_t tiles = (int64_t)((p.M + T - 1) / T) * (int64_t)((p.N + T - 1) / T);
        if (splits > 1) {
            ctr_off[j] = counters;
            counters += (size_t)tiles * kTcGroupCountersPerTile * sizeof(unsigned);
            part_off[j] = partials;
            partials += align256(tc_group_partial_floats(tiles, splits) * sizeof(float));
        }
    }
    // A operands that TMA cannot read in place: one zero-padded buffer, rows
    // of a multiple of 4 floats; the padding is never written and stays zero
    // (the tensor maps' K bounds the loads in any case).
    std::vector<size_t> pad_off(n, SIZE_MAX);
    size_t pad_bytes = 0;
    for (size_t j = 0; j < n; j++) {
        const maxmulsk_problem& p = problems[idx[j]];
        if (p.K % 4 == 0 && (uintptr_t)p.A % 16 == 0) continue;
        pad_off[j] = pad_bytes;
        pad_bytes += align256((size_t)p.M * ((p.K + 3) / 4 * 4) * sizeof(float));
    }
    if (pad_bytes) {
        cudaError_t e = cudaMalloc(&g->d_apad, pad_bytes);
        if (e == cudaSuccess) e = cudaMemset(g->d_apad, 0, pad_bytes);
        if (e != cudaSuccess) return cuda_status(e, "grouped: padded A buffer");
    }
    for (size_t j = 0; j < n; j++) {
        const maxmulsk_problem& p = problems[idx[j]];
        const float* a = p.A;
        int64_t lda = (int64_t)p.K;
        if (pad_off[j] != SIZE_MAX) {
            float* dst = reinterpret_cast<float*>(static_cast<char*>(g->d_apad) + pad_off[j]);
            lda = (int64_t)((p.K + 3) / 4 * 4);
            g->repack.push_back({dst, p.A, p.M, p.K, (size_t)lda});
            a = dst;
        }
        if (!tc_fused_maps(a, lda, p.B, (int64_t)p.M, (int64_t)p.K, (int64_t)p.N, &maps[256 * j])) {
            set_error_message("grouped: tensor map encoding failed");
            return MAXMULSK_ERR_CUDA;
        }
    }
    const size_t probs_b = align256(std::max<size_t>(1, n) * sizeof(TcGroupProblem));
    // units are counted below; reserve after building them
    g->tc_counter_bytes = align256(counters);
    for (size_t j = 0; j < n; j++) {
        const maxmulsk_problem& p = problems[idx[j]];
        TcGroupProblem& q = hp[j];
        std::memset(&q, 0, sizeof q);
        q.M = (int64_t)p.M; q.K = (int64_t)p.K; q.N = (int64_t)p.N;
        q.C = p.C;
        q.splits = slice_count(p.K, sk[j]);
        q.kchunk = (int64_t)slice_len(p.K, sk[j]);
        q.tiles_n = (int32_t)((p.N + T - 1) / T);
        q.chunk_kb = tc_chunk_len((int64_t)p.K, q.splits) / 32;
        const int tm_n = (int)((p.M + T - 1) / T);
        for (int z = 0; z < q.splits; z++)
            for (int tm = 0; tm < tm_n; tm++)
                for (int tn = 0; tn < q.tiles_n; tn++) hu.push_back(TcGroupUnit{(int32_t)j, tm, tn, z});
    }
    std::stable_sort(hu.begin(), hu.end(), [&](const TcGroupUnit& x, const TcGroupUnit& y) {
        const TcGroupProblem& a = hp[x.problem];
        const TcGroupProblem& b = hp[y.problem];
        const int64_t la = std::min(a.kchunk, a.K - (int64_t)x.z * a.kchunk);
        const int64_t lb = std::min(b.kchunk, b.K - (int64_t)y.z * b.kchunk);
        return la > lb;
    });
    const size_t units_b = align256(std::max<size_t>(1, hu.size()) * sizeof(TcGroupUnit));
    const size_t maps_b = align256(maps.size());
    const size_t total = probs_b + units_b + maps_b + g->tc_counter_bytes + partials;
    cudaError_t e = cudaMalloc(&g->d_tc, total);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(grouped tensor-core tables)");
    char* base = static_cast<char*>(g->d_tc);
    char* d_probs = base;
    char* d_units = d_probs + probs_b;
    char* d_maps = d_units + units_b;
    char* d_ctr = d_maps + maps_b;
    char* d_part = d_ctr + g->tc_counter_bytes;
    for (size_t j = 0; j < n; j++) {
        if (hp[j].splits > 1) {
            hp[j].counters = reinterpret_cast<unsigned*>(d_ctr + ctr_off[j]);
            hp[j].partial = reinterpret_cast<float*>(d_part + part_off[j]);
        }
    }
    if ((e = cudaMemcpy(d_probs, hp.data(), n * sizeof(TcGroupProblem), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (!hu.empty() && (e = cudaMemcpy(d_units, hu.data(), hu.size() * sizeof(TcGroupUnit),
                                        cudaMemcpyHostToDevice)) != cudaSuccess) ||
        (e = cudaMemcpy(d_maps, maps.data(), 256 * n, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_status(e, "upload grouped tensor-core tables");
    g->tc_counters = d_ctr;
    g->tc.probs = reinterpret_cast<const TcGroupProblem*>(d_probs);
    g->tc.units = reinterpret_cast<const TcGroupUnit*>(d_units);
    g->tc.maps = d_maps;
    g->tc.nunits = (int64_t)hu.size();
    g->tc.err = device_error_word();
    g->tc.timeout = 2000000000LL;                             // about one second at B200 clocks
    g->tc_grid = (int)std::max<int64_t>(1, std::min<int64_t>(g->tc.nunits, sms));
    if (!g->tc.err) { set_error_message("device error word unavailable"); return MAXMULSK_ERR_ALLOC; }
    return MAXMULSK_OK;
}

// B is read in place by TMA; A, if it cannot be, is repacked (build_tc).
bool fused_readable(const maxmulsk_problem& p) {
    return p.N % 4 == 0 && ((uintptr_t)p.B % 16) == 0;
}

// How a group is cut into work (one candidate of the configuration search).
struct GroupConfig {
    maxmulsk_plan simt{};          // FP32 part: tile, variant; split_k > 0 = that split for all
    double simt_share = 4.0;       // FP32 K-split policy (plan_splits) when split_k == 0
    int tc_precision = 0;          // 0: FP32 group; else BF16X6 / BF16X9 (the fused kernel)
    int tc_request = 0;            // the precision asked for (SPLIT_AUTO lets singles pick 3xTF32)
    int tc_fixed = 0;              // > 0: that split for every fused problem
    double tc_share = 4.0;
    double single_gflop = INFINITY;
};

// Split-precision problems that run as their own launches under `cfg`.
void pick_singles(const maxmulsk_problem* problems, std::vector<size_t>& tc_idx, const GroupConfig& cfg, int sms,
                  std::vector<maxmulsk_grouped_s::Single>& singles) {
    if (!(cfg.single_gflop < INFINITY)) return;
    std::vector<size_t> keep;
    for (size_t i : tc_idx) {
        const maxmulsk_problem& p = problems[i];
        const double gflop = 2.0 * (double)p.M * (double)p.N * (double)p.K * 1e-9;
        if (gflop >= cfg.single_gflop) {
            const maxmulsk_plan pl = choose_tuned(p.M, p.K, p.N, cfg.tc_request, sms);
            if (pl.precision != MAXMULSK_PREC_FP32 && pl.variant != MAXMULSK_TC_FUSED_SPLIT &&
                classify_plan(p.M, p.K, p.N, &pl) == MAXMULSK_OK) {
                singles.push_back({i, pl});
                continue;
            }
        }
        keep.push_back(i);
    }
    tc_idx.swap(keep);
}

// Plans, tables and scratch of one configuration (no capture yet).
maxmulsk_status build_group(maxmulsk_grouped_s* g, const maxmulsk_problem* problems, size_t count,
                            const GroupConfig& cfg, int sms) {
    g->count = count;
    g->split_k.assign(count, 1);
    g->plans.assign(count, maxmulsk_plan{});
    std::vector<size_t> simt_idx, tc_idx;
    for (size_t i = 0; i < count; i++) {
        if (cfg.tc_precision && runs(problems[i]) && fused_readable(problems[i])) tc_idx.push_back(i);
        else simt_idx.push_back(i);
    }
    pick_singles(problems, tc_idx, cfg, sms, g->singles);
    g->simt_plan = cfg.simt;
    if (cfg.tc_precision) {
        std::memset(&g->plan, 0, sizeof g->plan);
        g->plan.precision = cfg.tc_precision; g->plan.tile_m = 128; g->plan.tile_n = 128;
        g->plan.split_k = cfg.tc_fixed; g->plan.variant = MAXMULSK_TC_FUSED_SPLIT;
    } else {
        g->plan = cfg.simt;
    }
    maxmulsk_status st = build_simt(g, problems, simt_idx, cfg.simt, cfg.simt_share, sms);
    if (st == MAXMULSK_OK && !tc_idx.empty())
        st = build_tc(g, problems, tc_idx, cfg.tc_precision, cfg.tc_fixed, cfg.tc_share, sms);
    if (st != MAXMULSK_OK) return st;
    size_t ws = 0;
    for (const auto& sg : g->singles) {
        const maxmulsk_problem& p = problems[sg.problem];
        g->plans[sg.problem] = sg.plan;
        g->split_k[sg.problem] = sg.plan.split_k;
        ws = std::max(ws, workspace_bytes(p.M, p.K, p.N, sg.plan));
    }
    if (ws) {
        cudaError_t e = cudaMalloc(&g->d_single_ws, ws);
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(grouped single-launch workspace)");
        g->single_ws_bytes = ws;
    }
    return MAXMULSK_OK;
}

// Captures the group's work into its graph: K == 0 problems zero-filled, the
// unit counter and split-K arrival counters reset, the A repacks, the
// persistent kernel(s), then the single launches.
maxmulsk_status capture_group(maxmulsk_grouped_s* g, const maxmulsk_problem* problems) {
    cudaError_t e = cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamCreate");
    maxmulsk_status st = MAXMULSK_OK;
    e = cudaStreamBeginCapture(g->cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (size_t i = 0; i < g->count; i++)
            if (problems[i].M && problems[i].N && !problems[i].K)
                cudaMemsetAsync(problems[i].C, 0, problems[i].M * problems[i].N * sizeof(float), g->cap);
        if (g->tc_counters && g->tc_counter_bytes) cudaMemsetAsync(g->tc_counters, 0, g->tc_counter_bytes, g->cap);
        for (const auto& r : g->repack) {
            cudaError_t ec = cudaMemcpy2DAsync(r.dst, r.dst_ld * sizeof(float), r.src, r.cols * sizeof(float),
                                               r.cols * sizeof(float), r.rows, cudaMemcpyDeviceToDevice, g->cap);
            if (ec != cudaSuccess) e = ec;
        }
        if (g->tc.nunits > 0) {
            cudaError_t el = tc_grouped_launch(g->tc, g->plan.precision, g->tc_grid, g->cap);
            if (el != cudaSuccess) e = el;
        }
        cudaMemsetAsync(g->d_next, 0, sizeof(unsigned), g->cap);
        if (g->d_scratch && g->counter_bytes) cudaMemsetAsync(g->d_scratch, 0, g->counter_bytes, g->cap);
        if (g->nunits > 0)
            simt_grouped_launch(g->d_probs, g->d_units, g->nunits, g->d_next, g->simt_plan.tile_m,
                                g->simt_plan.tile_n, g->simt_plan.variant, g->grid, g->cap);
        for (const auto& sg : g->singles) {
            const maxmulsk_problem& p = problems[sg.problem];
            maxmulsk_status s1 = run_plan_dev(p.A, p.B, p.C, p.M, p.K, p.N, sg.plan, g->d_single_ws,
                                              g->single_ws_bytes, g->cap);
            if (s1 != MAXMULSK_OK && st == MAXMULSK_OK) st = s1;
        }
        cudaError_t e2 = cudaStreamEndCapture(g->cap, &g->graph);
        if (e == cudaSuccess) e = e2;
    }
    if (e == cudaSuccess && st == MAXMULSK_OK) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (st != MAXMULSK_OK) return st;
    return cuda_status(e, "grouped graph capture");
}

// Median of three timed replays of the group's graph (after one warm
// replay), in milliseconds; +inf if a replay fails.
float time_group(maxmulsk_grouped_s* g) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return INFINITY;
    }
    float t[3] = {INFINITY, INFINITY, INFINITY};
    cudaError_t e = cudaGraphLaunch(g->exec, g->cap);
    for (int i = 0; i < 3 && e == cudaSuccess; i++) {
        cudaEventRecord(e0, g->cap);
        e = cudaGraphLaunch(g->exec, g->cap);
        cudaEventRecord(e1, g->cap);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) cudaEventElapsedTime(&t[i], e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess || stream_status(g->cap) != MAXMULSK_OK) return INFINITY;
    std::sort(t, t + 3);
    return t[1];
}

// The candidates searched when the caller leaves the cut to the library.
std::vector<GroupConfig> candidate_configs(const GroupConfig& base, bool search_tile, bool search_simt,
                                           bool search_tc) {
    const int tiles[3][2] = {{128, 128}, {128, 64}, {64, 64}};
    const double shares[4] = {0.0, 2.0, 4.0, 8.0};            // 0: no K split
    std::vector<GroupConfig> simt_opts;
    if (search_simt) {
        for (int t = 0; t < (search_tile ? 3 : 1); t++)
            for (double sh : shares) {
                GroupConfig c = base;
                if (search_tile) { c.simt.tile_m = tiles[t][0]; c.simt.tile_n = tiles[t][1]; }
                c.simt_share = sh;
                simt_opts.push_back(c);
            }
    } else {
        simt_opts.push_back(base);
    }
    if (!base.tc_precision || !search_tc) return simt_opts;
    // Split-precision groups: the FP32 part (problems the fused split cannot
    // read) keeps the first option; the search runs over the rest.
    std::vector<GroupConfig> out;
    const double tc_shares[3] = {2.0, 4.0, 8.0};
    const double singles[4] = {INFINITY, 32.0, 8.0, 2.0};
    for (double th : singles)
        for (double sh : tc_shares) {
            GroupConfig c = simt_opts.front();
            c.tc_share = sh;
            c.single_gflop = th;
            out.push_back(c);
        }
    return out;
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
    GroupConfig base;
    std::memset(&base.simt, 0, sizeof base.simt);
    base.simt.precision = MAXMULSK_PREC_FP32;
    base.simt.variant = MAXMULSK_FP32_FMA;
    bool search_tile = true, search_simt = true, search_tc = false;
    const int sms = device_sm_count() > 0 ? device_sm_count() : 148;
    std::vector<size_t> all(count);
    for (size_t i = 0; i < count; i++) all[i] = i;
    if (group_plan) {
        const maxmulsk_plan plan = *group_plan;
        if (plan.split_k < 0 || plan.split_k > 64) {
            set_error_message("split_k must be 0 (chosen by the library) or 1..64");
            return MAXMULSK_ERR_UNSUPPORTED;
        }
        if (plan.precision == MAXMULSK_PREC_SPLIT_AUTO || plan.precision == MAXMULSK_PREC_BF16X6 ||
            plan.precision == MAXMULSK_PREC_BF16X9) {
            base.tc_request = plan.precision;
            base.tc_precision = plan.precision == MAXMULSK_PREC_BF16X9 ? MAXMULSK_PREC_BF16X9 : MAXMULSK_PREC_BF16X6;
            base.tc_fixed = plan.split_k;
            search_tc = plan.split_k == 0;
            // problems the fused split cannot read: FP32, tile by padded work, split by the formula
            std::vector<size_t> fp32_idx;
            for (size_t i = 0; i < count; i++)
                if (!(runs(problems[i]) && fused_readable(problems[i]))) fp32_idx.push_back(i);
            pick_tile(problems, fp32_idx, &base.simt.tile_m, &base.simt.tile_n);
            search_tile = search_simt = false;
        } else if (plan.precision != MAXMULSK_PREC_FP32) {
            set_error_message("grouped launches run FP32, BF16X6, BF16X9 or SPLIT_AUTO plans");
            return MAXMULSK_ERR_UNSUPPORTED;
        } else {
            maxmulsk_plan probe = plan;
            if (probe.split_k == 0) probe.split_k = 1;
            maxmulsk_status st = classify_plan(1, 1, 1, &probe);
            if (st != MAXMULSK_OK) return st;
            base.simt.tile_m = plan.tile_m; base.simt.tile_n = plan.tile_n; base.simt.variant = plan.variant;
            base.simt.split_k = plan.split_k;
            search_tile = false;
            search_simt = plan.split_k == 0;
        }
    } else {
        pick_tile(problems, all, &base.simt.tile_m, &base.simt.tile_n);
    }

    const std::vector<GroupConfig> cands = candidate_configs(base, search_tile, search_simt, search_tc);
    std::unique_ptr<maxmulsk_grouped_s> best;
    float best_ms = INFINITY;
    maxmulsk_status last = MAXMULSK_OK;
    for (const GroupConfig& cfg : cands) {
        std::unique_ptr<maxmulsk_grouped_s> g(new (std::nothrow) maxmulsk_grouped_s());
        if (!g) return MAXMULSK_ERR_ALLOC;
        cudaGetDevice(&g->device);
        maxmulsk_status st = build_group(g.get(), problems, count, cfg, sms);
        if (st == MAXMULSK_OK) st = capture_group(g.get(), problems);
        if (st != MAXMULSK_OK) {
            last = st;
            maxmulsk_grouped_destroy(g.release());
            continue;
        }
        const float ms = cands.size() > 1 ? time_group(g.get()) : 0.0f;
        if (!best || ms < best_ms) {
            if (best) maxmulsk_grouped_destroy(best.release());
            best = std::move(g);
            best_ms = ms;
        } else {
            maxmulsk_grouped_destroy(g.release());
        }
    }
    if (!best) return last != MAXMULSK_OK ? last : MAXMULSK_ERR_UNSUPPORTED;
    *out = best.release();
    return MAXMULSK_OK;
}

maxmulsk_status maxmulsk_grouped_launch(maxmulsk_grouped g, void* stream) {
    if (!g || !g->exec) return MAXMULSK_ERR_INVALID;
    PhaseScope ps(kPhaseGrouped, static_cast<cudaStream_t>(stream));
    return cuda_status(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch(grouped)");
}

maxmulsk_status maxmulsk_grouped_info(maxmulsk_grouped g, maxmulsk_plan* group_plan, int32_t* split_k,
                                      size_t* units) {
    if (!g) return MAXMULSK_ERR_INVALID;
    if (group_plan) *group_plan = g->plan;
    if (split_k) std::memcpy(split_k, g->split_k.data(), g->count * sizeof(int32_t));
    if (units) *units = (size_t)g->nunits + (size_t)g->tc.nunits + g->singles.size();
    return MAXMULSK_OK;
}

maxmulsk_status maxmulsk_grouped_plans(maxmulsk_grouped g, maxmulsk_plan* plans) {
    if (!g || (!plans && g->count)) return MAXMULSK_ERR_INVALID;
    if (g->count) std::memcpy(plans, g->plans.data(), g->count * sizeof(maxmulsk_plan));
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
    cudaFree(g->d_tc);
    cudaFree(g->d_apad);
    cudaFree(g->d_single_ws);
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
