// Tuning database: measured best plan per exact shape.
//
// The reference keeps a static shape -> Blocking table compiled into the
// library, square shapes only, each entry justified by repeated measurement
// (sme/support/gemm_tuning.cpp:34-37, rules at sme/support/gemm_tuning.hpp:8-24).
// Here the table is data: a text file written by the autotuner, one line per
// (M, K, N, requested precision):
//     M K N requested precision tile_m tile_n split_k variant time_us
// (`requested` is the precision argument of the call; `precision` the plan's,
// which differs for MAXMULSK_PREC_SPLIT_AUTO).
// Lines starting with '#' are comments. Loaded once (MAXMULSK_TUNING_DB) under
// a mutex; lookups take the same mutex.
#include "tuning.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "mlp.hpp"

namespace mmsk {

namespace {
using Key = std::tuple<size_t, size_t, size_t, int>;
struct Entry { maxmulsk_plan plan; double time_us; };

std::mutex g_mu;
std::map<Key, Entry> g_db;
bool g_env_loaded = false;

int load_locked(const char* path) {
    FILE* f = std::fopen(path, "r");
    if (!f) return -1;
    char line[512];
    int n = 0;
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        unsigned long long M, K, N;
        int key, prec, tm, tn, sk, var;
        double t;
        if (std::sscanf(line, "%llu %llu %llu %d %d %d %d %d %d %lf", &M, &K, &N, &key, &prec, &tm, &tn, &sk, &var,
                        &t) != 10)
            continue;
        maxmulsk_plan p;
        std::memset(&p, 0, sizeof p);
        p.precision = prec; p.tile_m = tm; p.tile_n = tn; p.split_k = sk; p.variant = var;
        g_db[Key{(size_t)M, (size_t)K, (size_t)N, key}] = Entry{p, t};
        n++;
    }
    std::fclose(f);
    return n;
}

void ensure_env_loaded_locked() {
    if (g_env_loaded) return;
    g_env_loaded = true;
    const char* path = std::getenv("MAXMULSK_TUNING_DB");
    if (path && *path) load_locked(path);
}
}  // namespace

bool tuning_lookup(size_t M, size_t K, size_t N, int precision, maxmulsk_plan* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    ensure_env_loaded_locked();
    auto it = g_db.find(Key{M, K, N, precision});
    if (it == g_db.end()) return false;
    *out = it->second.plan;
    return true;
}

bool tuning_predict(size_t M, size_t K, size_t N, int precision, maxmulsk_plan* out) {
    return mlp_predict_plan(M, K, N, precision, out);
}

int tuning_load_db(const char* path) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_env_loaded = true;
    g_db.clear();
    return load_locked(path);
}

void tuning_put(size_t M, size_t K, size_t N, int key, const maxmulsk_plan& p, double time_us) {
    std::lock_guard<std::mutex> lk(g_mu);
    ensure_env_loaded_locked();
    g_db[Key{M, K, N, key}] = Entry{p, time_us};
}

int tuning_save_db(const char* path) {
    std::lock_guard<std::mutex> lk(g_mu);
    FILE* f = std::fopen(path, "w");
    if (!f) return -1;
    std::fprintf(f, "# maxmulsk tuning database: M K N requested precision tile_m tile_n split_k variant time_us\n");
    int n = 0;
    for (const auto& kv : g_db) {
        const auto& k = kv.first;
        const auto& e = kv.second;
        std::fprintf(f, "%zu %zu %zu %d %d %d %d %d %d %.3f\n", std::get<0>(k), std::get<1>(k), std::get<2>(k),
                     std::get<3>(k), e.plan.precision, e.plan.tile_m, e.plan.tile_n, e.plan.split_k, e.plan.variant,
                     e.time_us);
        n++;
    }
    std::fclose(f);
    return n;
}

void tuning_clear() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_env_loaded = true;
    g_db.clear();
}

}  // namespace mmsk

extern "C" {
int32_t maxmulsk_tuning_load(const char* path) { return path ? mmsk::tuning_load_db(path) : -1; }
int32_t maxmulsk_tuning_save(const char* path) { return path ? mmsk::tuning_save_db(path) : -1; }
void maxmulsk_tuning_clear(void) { mmsk::tuning_clear(); }
}
