// transcript.h -- Fiat-Shamir transcript: Poseidon2 (width 8) overwrite sponge.
//
// Sponge semantics follow Poseidon2Transcript
// (crates/neo-transcript/src/poseidon2.rs:10-310): rate 4, overwrite absorb,
// labels and lengths absorbed one field element per byte, challenge_field =
// append_message("chal/label", label) + absorb(1) + permute + st[0].
//
// The permutation is Poseidon2 (Grassi, Khovratovich, Schofnegger, eprint
// 2023/323) over Goldilocks, t = 8, x^7 S-box, R_F = 8, R_P = 22, external
// layer circ(2 M4, M4) with the paper's M4, internal layer 1 + diag(mu).  Round
// constants and mu are drawn from ChaCha8 (RFC 7539 block function with 8
// rounds) seeded with SEED = "neo_poseidon2_goldilocks_seed___"
// (crates/neo-params/src/poseidon2_goldilocks.rs:61) by rejection sampling
// u64 < q.  The reference takes its constants from the un-vendored
// p3-poseidon2 0.4.1 new_from_rng_128; whether this derivation matches it is
// not verifiable here, so transcript states are parity-unpinned.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace neo {

struct ChaCha8 {
    uint32_t key[8];
    uint64_t counter = 0;
    uint32_t block[16];
    int idx = 16;
    explicit ChaCha8(const uint8_t seed[32]);
    uint32_t next_u32();
    uint64_t next_u64();
    void fill_bytes(uint8_t* out, size_t n);

   private:
    void refill();
};

// rand_core's documented seed_from_u64 expansion: a PCG32 (XSH-RR) stream
// fills the 32-byte seed 4 bytes at a time.
void seed_from_u64(uint64_t state, uint8_t seed[32]);

// Poseidon2 over Goldilocks with width W in {8, 16}.
template <int W>
struct Poseidon2 {
    static constexpr int RF = 8, RP = 22;
    uint64_t rc_ext[RF][W];
    uint64_t rc_int[RP];
    uint64_t mu[W];  // internal diagonal: M_I x = sum(x) + mu_i * x_i
    explicit Poseidon2(const uint8_t seed[32]);
    void permute(uint64_t* st) const;
};
using Poseidon2W8 = Poseidon2<8>;
using Poseidon2W16 = Poseidon2<16>;
// the transcript permutation (seeded with the reference SEED)
const Poseidon2W8& transcript_perm();
// the CCS-digest permutation (ChaCha8Rng::seed_from_u64(0x434353445F4D4154))
const Poseidon2W16& digest_perm();

class Transcript {
   public:
    static constexpr int RATE = 4;
    explicit Transcript(const std::string& app_label);
    void append_message(const std::string& label, const uint8_t* msg, size_t len);
    void append_message(const std::string& label, const std::string& msg) {
        append_message(label, reinterpret_cast<const uint8_t*>(msg.data()), msg.size());
    }
    void append_fields(const std::string& label, const uint64_t* fs, size_t n);
    void append_u64s(const std::string& label, const uint64_t* us, size_t n);
    uint64_t challenge_field(const std::string& label);
    void challenge_fields(const std::string& label, size_t n, uint64_t* out);
    void digest32(uint8_t out[32]);
    const uint64_t* state() const { return st_; }
    uint64_t permutations() const { return perms_; }
    // the whole sponge position, for checkpointing a prover and resuming it
    void save(uint64_t st[8], uint32_t* absorbed, uint64_t* perms) const {
        memcpy(st, st_, sizeof st_);
        *absorbed = (uint32_t)absorbed_;
        *perms = perms_;
    }
    bool restore(const uint64_t st[8], uint32_t absorbed, uint64_t perms) {
        if (absorbed > (uint32_t)RATE) return false;
        memcpy(st_, st, sizeof st_);
        absorbed_ = (int)absorbed;
        perms_ = perms;
        return true;
    }

   private:
    void absorb_elem(uint64_t x);
    void absorb_slice(const uint64_t* xs, size_t n);
    void absorb_label(const std::string& label);
    void permute();
    uint64_t st_[8];
    int absorbed_ = 0;
    uint64_t perms_ = 0;
};

}  // namespace neo
