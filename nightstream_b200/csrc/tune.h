// tune.h -- launch choices of the Pi_CCS row rounds per (ell_n, k) (tune.cu).
#pragma once
#include <cstdint>

struct CcsTune {
    uint64_t nc_threads;  // NC threads per round (rounds >= 3)
    uint32_t compact_q;   // q per thread below which K products are out of line
    uint32_t hist_items;  // target items per histogram block
};

bool tune_lookup(uint32_t ell, uint32_t k, CcsTune* out);
void tune_store(uint32_t ell, uint32_t k, const CcsTune& t);
// Forces the choice of this thread's next oracle initialisations (nullptr: off).
void tune_force(const CcsTune* t);
