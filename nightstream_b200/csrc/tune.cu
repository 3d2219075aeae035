// tune.cu -- launch-shape autotuner for the Pi_CCS row rounds.
//
// The ternary-digit rounds (ccs_fast.cuh) have three launch choices whose best
// value depends on the shape (ell_n rows, k digit witnesses) and the GPU:
//   nc_threads  threads of the NC blocks per round (rounds >= 3),
//   compact_q   q per thread below which those blocks call out-of-line K products,
//   hist_items  (q, 8-row block) items per histogram block (round 0).
// A process-wide table maps (ell_n, k) to the best choice.  neo_gpu_ccs_autotune
// times the whole row-round sequence of a caller's oracle inputs for every
// candidate (CUDA events, random challenges) and records the fastest;
// neo_gpu_tune_save / neo_gpu_tune_load keep the table in a text file (one
// line "ccs <ell_n> <k> <nc_threads> <compact_q> <hist_items>" per shape), so
// a table measured once on the target GPU ships with the library.
#include "internal.cuh"
#include <cstdio>
#include <map>
#include <mutex>

#include "tune.h"

namespace {
std::mutex g_tune_mu;
std::map<std::pair<uint32_t, uint32_t>, CcsTune> g_tune;
thread_local const CcsTune* g_forced = nullptr;
}  // namespace

bool tune_lookup(uint32_t ell, uint32_t k, CcsTune* out) {
    if (g_forced) {
        *out = *g_forced;
        return true;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({ell, k});
    if (it == g_tune.end()) return false;
    *out = it->second;
    return true;
}

void tune_store(uint32_t ell, uint32_t k, const CcsTune& t) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{ell, k}] = t;
}

void tune_force(const CcsTune* t) { g_forced = t; }

static int neo_gpu_tune_load_impl_abi(const char* path) {
    if (!path) return NEO_ERR_ARG;
    FILE* f = fopen(path, "r");
    if (!f) return NEO_ERR_ARG;
    char kind[16];
    unsigned ell, k, cq, hi;
    unsigned long long nt;
    while (fscanf(f, "%15s %u %u %llu %u %u", kind, &ell, &k, &nt, &cq, &hi) == 6) {
        if (std::string(kind) != "ccs" || ell > 30 || k == 0 || nt == 0 || hi == 0) continue;
        tune_store(ell, k, CcsTune{nt, cq, hi});
    }
    fclose(f);
    return NEO_OK;
}
extern "C" int neo_gpu_tune_load(const char* path) { NEO_ABI_GUARD(neo_gpu_tune_load_impl_abi(path)) }

static int neo_gpu_tune_save_impl_abi(const char* path) {
    if (!path) return NEO_ERR_ARG;
    FILE* f = fopen(path, "w");
    if (!f) return NEO_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto& e : g_tune)
        fprintf(f, "ccs %u %u %llu %u %u\n", e.first.first, e.first.second, (unsigned long long)e.second.nc_threads,
                e.second.compact_q, e.second.hist_items);
    fclose(f);
    return NEO_OK;
}
extern "C" int neo_gpu_tune_save(const char* path) { NEO_ABI_GUARD(neo_gpu_tune_save_impl_abi(path)) }

static int neo_gpu_tune_get_impl_abi(uint32_t ell_n, uint32_t k, uint64_t* out3) {
    if (!out3) return NEO_ERR_ARG;
    CcsTune t;
    if (!tune_lookup(ell_n, k, &t)) return NEO_ERR_ARG;
    out3[0] = t.nc_threads;
    out3[1] = t.compact_q;
    out3[2] = t.hist_items;
    return NEO_OK;
}
extern "C" int neo_gpu_tune_get(uint32_t ell_n, uint32_t k, uint64_t* out3) { NEO_ABI_GUARD(neo_gpu_tune_get_impl_abi(ell_n, k, out3)) }
