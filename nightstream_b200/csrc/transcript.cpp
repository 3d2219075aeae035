// transcript.cpp -- Poseidon2 width-8 permutation, ChaCha8 and the sponge.
#include "transcript.h"
#include <cstdlib>
#include "gl.cuh"
#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace neo {

// ---------------------------------------------------------------- ChaCha8 --
static inline uint32_t rotl(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }
#define QR(a, b, c, d)          \
    a += b; d ^= a; d = rotl(d, 16); \
    c += d; b ^= c; b = rotl(b, 12); \
    a += b; d ^= a; d = rotl(d, 8);  \
    c += d; b ^= c; b = rotl(b, 7);

ChaCha8::ChaCha8(const uint8_t seed[32]) {
    for (int i = 0; i < 8; i++)
        key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                 ((uint32_t)seed[4 * i + 3] << 24);
}

void ChaCha8::refill() {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                      key[4],      key[5],      key[6],      key[7],      (uint32_t)counter,
                      (uint32_t)(counter >> 32), 0u, 0u};
    uint32_t x[16];
    memcpy(x, s, sizeof x);
    for (int r = 0; r < 4; r++) {  // 8 rounds = 4 double rounds
        QR(x[0], x[4], x[8], x[12]);
        QR(x[1], x[5], x[9], x[13]);
        QR(x[2], x[6], x[10], x[14]);
        QR(x[3], x[7], x[11], x[15]);
        QR(x[0], x[5], x[10], x[15]);
        QR(x[1], x[6], x[11], x[12]);
        QR(x[2], x[7], x[8], x[13]);
        QR(x[3], x[4], x[9], x[14]);
    }
    for (int i = 0; i < 16; i++) block[i] = x[i] + s[i];
    counter++;
    idx = 0;
}

uint32_t ChaCha8::next_u32() {
    if (idx >= 16) refill();
    return block[idx++];
}
uint64_t ChaCha8::next_u64() {
    uint64_t lo = next_u32();
    uint64_t hi = next_u32();
    return lo | (hi << 32);
}
void ChaCha8::fill_bytes(uint8_t* out, size_t n) {
    size_t i = 0;
    while (i < n) {
        uint32_t w = next_u32();
        for (int b = 0; b < 4 && i < n; b++, i++) out[i] = (uint8_t)(w >> (8 * b));
    }
}

// --------------------------------------------------------------- Poseidon2 --
static const uint8_t SEED[32] = {'n', 'e', 'o', '_', 'p', 'o', 's', 'e', 'i', 'd', 'o', 'n', '2', '_', 'g', 'o',
                                 'l', 'd', 'i', 'l', 'o', 'c', 'k', 's', '_', 's', 'e', 'e', 'd', '_', '_', '_'};

static uint64_t sample_fq(ChaCha8& rng) {
    for (;;) {
        uint64_t x = rng.next_u64();
        if (x < GL_Q) return x;
    }
}

void seed_from_u64(uint64_t state, uint8_t seed[32]) {
    const uint64_t MUL = 6364136223846793005ULL, INC = 11634580027462260723ULL;
    for (int c = 0; c < 8; c++) {
        state = state * MUL + INC;
        uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        uint32_t x = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
        for (int b = 0; b < 4; b++) seed[4 * c + b] = (uint8_t)(x >> (8 * b));
    }
}

template <int W>
Poseidon2<W>::Poseidon2(const uint8_t seed[32]) {
    ChaCha8 rng(seed);
    for (int r = 0; r < RF; r++)
        for (int i = 0; i < W; i++) rc_ext[r][i] = sample_fq(rng);
    for (int r = 0; r < RP; r++) rc_int[r] = sample_fq(rng);
    for (int i = 0; i < W; i++) mu[i] = sample_fq(rng);
}

const Poseidon2W8& transcript_perm() {
    static const Poseidon2W8 inst(SEED);
    return inst;
}

const Poseidon2W16& digest_perm() {
    static const Poseidon2W16 inst([] {
        static uint8_t s[32];
        seed_from_u64(0x434353445F4D4154ULL, s);
        return (const uint8_t*)s;
    }());
    return inst;
}

typedef unsigned __int128 u128;

// Permutation arithmetic keeps lanes in [0, 2^64) (not necessarily < q) and
// canonicalises once at the end. The transcript is one sequential chain of
// permutations, so every reduction is written for latency:
//  * a + b with carry: 2^64 = 2^32 - 1 (mod q), so the correction is the
//    carry widened to 32 ones, which `sbb` on a 32-bit register produces
//    directly (add, sbb, add);
//  * lo - hi_hi borrows only when lo < hi_hi < 2^32, i.e. with probability
//    about 2^-32 for a product, so it is a branch the predictor never misses
//    instead of a mask on the critical path.
// State loops are fully unrolled so the independent S-box chains of a full
// round overlap.
static inline __attribute__((always_inline)) uint64_t add_carry_fix(uint64_t a, uint64_t b) {
#if defined(__x86_64__)
    uint64_t adj;
    __asm__("add %[b], %[a]\n\tsbb %k[adj], %k[adj]\n\tadd %[adj], %[a]"
            : [a] "+r"(a), [adj] "=&r"(adj)
            : [b] "r"(b)
            : "cc");
    return a;
#else
    uint64_t s;
    const uint64_t c = __builtin_add_overflow(a, b, &s);
    return s + (GL_EPS & (0 - c));
#endif
}
static inline __attribute__((always_inline)) uint64_t red_nc(uint64_t lo, uint64_t hi) {
    // lo + 2^64 hi with 2^64 = 2^32 - 1 and 2^96 = -1 (mod q)
    const uint64_t hh = hi >> 32, hl = hi & GL_EPS;
    uint64_t t0;
    if (__builtin_expect(__builtin_sub_overflow(lo, hh, &t0), 0)) t0 -= GL_EPS;  // t0 >= 2^64 - 2^32 here
    // t0 + hl (2^32 - 1); a carry leaves a sum below hl (2^32 - 1), so the
    // correction cannot carry again
    return add_carry_fix(t0, (hl << 32) - hl);
}
static inline __attribute__((always_inline)) uint64_t red128(u128 x) { return red_nc((uint64_t)x, (uint64_t)(x >> 64)); }
// x with a high word below 2^32 (a sum of a few lanes): lo + hi (2^32 - 1)
static inline __attribute__((always_inline)) uint64_t red_small(u128 x) {
    const uint64_t hi = (uint64_t)(x >> 64);
    return add_carry_fix((uint64_t)x, (hi << 32) - hi);
}
static inline __attribute__((always_inline)) uint64_t mulq(uint64_t a, uint64_t b) { return red128((u128)a * b); }
// a + b for any a < 2^64 and b < q (a round constant): with a carry the sum
// a + b - 2^64 is below b < q = 2^64 - 2^32 + 1, so adding 2^32 - 1 cannot
// carry again
static inline __attribute__((always_inline)) uint64_t addq(uint64_t a, uint64_t b) { return add_carry_fix(a, b); }
static inline __attribute__((always_inline)) uint64_t canonq(uint64_t a) { return a >= GL_Q ? a - GL_Q : a; }

static inline __attribute__((always_inline)) uint64_t sbox7(uint64_t x) {
    const uint64_t x2 = mulq(x, x);
    const uint64_t x3 = mulq(x2, x);
    const uint64_t x4 = mulq(x2, x2);
    return mulq(x3, x4);
}

// M4 = [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] by the Poseidon2 paper's
// addition chain (8 additions, 4 doublings); inputs < 2^64, outputs < 2^69.
static inline __attribute__((always_inline)) void m4_lazy(const uint64_t* x, u128* y) {
    const u128 t0 = (u128)x[0] + x[1];
    const u128 t1 = (u128)x[2] + x[3];
    const u128 t2 = ((u128)x[1] << 1) + t1;
    const u128 t3 = ((u128)x[3] << 1) + t0;
    const u128 t4 = (t1 << 2) + t3;
    const u128 t5 = (t0 << 2) + t2;
    y[0] = t3 + t5;
    y[1] = t5;
    y[2] = t2 + t4;
    y[3] = t4;
}

// external layer circ(2 M4, M4, ..., M4): y_blk = M4 x_blk + sum_blk' M4 x_blk'
template <int W>
static inline __attribute__((always_inline)) void external_layer(uint64_t* st) {
    u128 y[W];
#pragma GCC unroll 4
    for (int b = 0; b < W / 4; b++) m4_lazy(st + 4 * b, y + 4 * b);
#pragma GCC unroll 4
    for (int i = 0; i < 4; i++) {
        u128 s = 0;
#pragma GCC unroll 4
        for (int b = 0; b < W / 4; b++) s += y[4 * b + i];
#pragma GCC unroll 4
        for (int b = 0; b < W / 4; b++) st[4 * b + i] = red_small(y[4 * b + i] + s);  // < 2^72
    }
}

// the S-box steps of all lanes are issued stage by stage (x^2, x^3, x^4, x^7)
// so the independent multiply chains interleave
template <int W>
static inline __attribute__((always_inline)) void full_round(uint64_t* st, const uint64_t* rc) {
    uint64_t x[W], x2[W], x3[W], x4[W];
#pragma GCC unroll 16
    for (int i = 0; i < W; i++) x[i] = addq(st[i], rc[i]);
#pragma GCC unroll 16
    for (int i = 0; i < W; i++) x2[i] = mulq(x[i], x[i]);
#pragma GCC unroll 16
    for (int i = 0; i < W; i++) x3[i] = mulq(x2[i], x[i]);
#pragma GCC unroll 16
    for (int i = 0; i < W; i++) x4[i] = mulq(x2[i], x2[i]);
#pragma GCC unroll 16
    for (int i = 0; i < W; i++) st[i] = mulq(x3[i], x4[i]);
    external_layer<W>(st);
}

template <int W>
__attribute__((noinline)) static void permute_impl(const Poseidon2<W>& P, uint64_t* st_io) {
    constexpr int RF = Poseidon2<W>::RF, RP = Poseidon2<W>::RP;
    uint64_t st[W];
#pragma GCC unroll 16
    for (int i = 0; i < W; i++) st[i] = st_io[i];
    external_layer<W>(st);
    for (int r = 0; r < RF / 2; r++) full_round<W>(st, P.rc_ext[r]);
    // Partial rounds: internal layer M_I x = sum(x) + mu_i * x_i.  Only lane 0
    // goes through the S-box, so with rest = Σ_{i>=1} x_i the new lane 0 is
    // (mu_0 + 1)·s + rest (one multiply-add after the S-box), while lanes
    // 1..W-1 and the next rest are computed beside the next S-box chain.  The
    // next round's constant joins that multiply-add (x0 is the S-box input),
    // which keeps a separate addition off the chain.
    u128 racc = 0;
#pragma GCC unroll 16
    for (int i = 1; i < W; i++) racc += st[i];
    uint64_t rest = red_small(racc);
    const uint64_t mu0p1 = P.mu[0] + 1;  // mu_0 < q, so no wrap
    uint64_t x0 = addq(st[0], P.rc_int[0]);
    for (int r = 0; r < RP; r++) {
        const uint64_t x = sbox7(x0);
        // both may lie in [q, 2^64), so the 65-bit sum goes through red_small
        // (addq is exact only when one operand is below q)
        const uint64_t sum = red_small((u128)x + rest);
        const u128 addend = (u128)rest + (r + 1 < RP ? P.rc_int[r + 1] : 0);
        x0 = red128((u128)mu0p1 * x + addend);  // < 2^128: mu0p1 < 2^64 - 2^32 + 2
        u128 nacc = 0;
#pragma GCC unroll 16
        for (int i = 1; i < W; i++) {
            st[i] = red128((u128)P.mu[i] * st[i] + sum);
            nacc += st[i];
        }
        rest = red_small(nacc);
    }
    st[0] = x0;
    for (int r = RF / 2; r < RF; r++) full_round<W>(st, P.rc_ext[r]);
#pragma GCC unroll 16
    for (int i = 0; i < W; i++) st_io[i] = canonq(st[i]);
}

#if defined(__x86_64__)
// --------------------------------------------------- width 16 on AVX-512 --
// The width-16 permutation (the CCS digest: a sponge over every nonzero of
// the matrices, five entries per permutation) is throughput-bound in scalar
// code: 16 independent S-boxes per full round and 15 linear lanes per
// partial round.  With the state in two zmm registers (8 x u64 each) both
// halves' multiply chains run side by side: full rounds do the S-boxes as
// 32 x 32 -> 64-bit partial products and the external layer on 32-bit lane
// halves (every intermediate fits 64 bits); partial rounds keep lane 0, the
// S-box chain, in scalar registers and lanes 1..15 in the vectors, whose next
// sum is sum_i mu_i x_i + 15 sum, so only lane 0's chain is serial.  Lanes
// stay in [0, 2^64) as in the scalar code and the result is bit-identical to
// it (1.5x faster on a Xeon with AVX-512).  These functions are also built
// for BMI2 (every AVX-512 CPU has it): the scalar products become mulx, whose
// free choice of registers saves the moves that mul's fixed rax/rdx operands
// cost (8 full width-8 rounds 295 -> 260 ns).  Width 8 keeps its full rounds
// scalar (eight S-box chains whose latency the vector multiply would lengthen)
// and moves lanes 1..7 of its partial rounds into one vector, beside lane 0's
// scalar chain (permute8_avx512).
#define NEO_AVX512 __attribute__((target("avx512f"), always_inline)) inline
NEO_AVX512 static __m512i v_eps() { return _mm512_set1_epi64((long long)GL_EPS); }
// (lo, hi) -> lo + 2^64 hi (mod q), the vector form of red_nc
NEO_AVX512 static __m512i v_red(__m512i lo, __m512i hi) {
    const __m512i eps = v_eps();
    const __m512i hh = _mm512_srli_epi64(hi, 32), hl = _mm512_and_si512(hi, eps);
    __m512i t0 = _mm512_sub_epi64(lo, hh);
    t0 = _mm512_mask_sub_epi64(t0, _mm512_cmplt_epu64_mask(lo, hh), t0, eps);
    const __m512i t1 = _mm512_sub_epi64(_mm512_slli_epi64(hl, 32), hl);
    const __m512i s = _mm512_add_epi64(t0, t1);
    return _mm512_mask_add_epi64(s, _mm512_cmplt_epu64_mask(s, t1), s, eps);
}
// a b (mod q) per lane from 32 x 32 -> 64 products: with a = ah 2^32 + al and
// b = bh 2^32 + bl, t = ah bl + (al bl >> 32) and u = al bh + (t mod 2^32)
// stay below 2^64, and a b = (al bl mod 2^32) + (u mod 2^32) 2^32
// + (ah bh + t / 2^32 + u / 2^32) 2^64.
NEO_AVX512 static __m512i v_mul(__m512i a, __m512i b, __m512i b_hi) {
    const __m512i m32 = v_eps();
    const __m512i a_hi = _mm512_srli_epi64(a, 32);
    const __m512i ll = _mm512_mul_epu32(a, b);
    const __m512i lh = _mm512_mul_epu32(a, b_hi);
    const __m512i hl = _mm512_mul_epu32(a_hi, b);
    const __m512i hh = _mm512_mul_epu32(a_hi, b_hi);
    const __m512i t = _mm512_add_epi64(hl, _mm512_srli_epi64(ll, 32));
    const __m512i u = _mm512_add_epi64(lh, _mm512_and_si512(t, m32));
    const __m512i lo = _mm512_or_si512(_mm512_slli_epi64(u, 32), _mm512_and_si512(ll, m32));
    const __m512i hi = _mm512_add_epi64(hh, _mm512_add_epi64(_mm512_srli_epi64(t, 32), _mm512_srli_epi64(u, 32)));
    return v_red(lo, hi);
}
NEO_AVX512 static __m512i v_mul(__m512i a, __m512i b) { return v_mul(a, b, _mm512_srli_epi64(b, 32)); }
// a + b with b < q in every lane (exact for the same reason as addq)
NEO_AVX512 static __m512i v_add_small(__m512i a, __m512i b) {
    const __m512i s = _mm512_add_epi64(a, b);
    return _mm512_mask_add_epi64(s, _mm512_cmplt_epu64_mask(s, b), s, v_eps());
}
// block-local M4 on lanes < 2^32: lane i is sum_k C_k[i] x[(i + k) mod 4]
// with C_0 = (5,6,5,6), C_1 = (7,1,7,1), C_2 = (1,1,1,1), C_3 = (3,4,3,4);
// outputs < 16 * 2^32
NEO_AVX512 static __m512i v_m4(__m512i v) {
    const __m512i r1 = _mm512_permutexvar_epi64(_mm512_set_epi64(4, 7, 6, 5, 0, 3, 2, 1), v);
    const __m512i r2 = _mm512_permutexvar_epi64(_mm512_set_epi64(5, 4, 7, 6, 1, 0, 3, 2), v);
    const __m512i r3 = _mm512_permutexvar_epi64(_mm512_set_epi64(6, 5, 4, 7, 2, 1, 0, 3), v);
    __m512i y = _mm512_mul_epu32(v, _mm512_set_epi64(6, 5, 6, 5, 6, 5, 6, 5));
    y = _mm512_add_epi64(y, _mm512_mul_epu32(r1, _mm512_set_epi64(1, 7, 1, 7, 1, 7, 1, 7)));
    y = _mm512_add_epi64(y, r2);
    return _mm512_add_epi64(y, _mm512_mul_epu32(r3, _mm512_set_epi64(4, 3, 4, 3, 4, 3, 4, 3)));
}
// lo + hi 2^32 (mod q) for lo, hi < 2^40: hi = a 2^32 + b, a 2^64 = a (2^32 - 1)
NEO_AVX512 static __m512i v_combine(__m512i lo, __m512i hi) {
    const __m512i m32 = v_eps();
    const __m512i a = _mm512_srli_epi64(hi, 32);
    const __m512i base = _mm512_add_epi64(lo, _mm512_sub_epi64(_mm512_slli_epi64(a, 32), a));
    const __m512i top = _mm512_slli_epi64(hi, 32);
    const __m512i s2 = _mm512_add_epi64(base, top);
    return _mm512_mask_add_epi64(s2, _mm512_cmplt_epu64_mask(s2, top), s2, m32);
}
// circ(2 M4, M4, M4, M4) with blocks 0, 1 in A and 2, 3 in B: the sum over
// blocks is the 256-bit-half swap of A + B; outputs < 2^39 per lane half
NEO_AVX512 static void v_external16(__m512i& A, __m512i& B) {
    const __m512i m32 = v_eps();
    const __m512i yal = v_m4(_mm512_and_si512(A, m32)), yah = v_m4(_mm512_srli_epi64(A, 32));
    const __m512i ybl = v_m4(_mm512_and_si512(B, m32)), ybh = v_m4(_mm512_srli_epi64(B, 32));
    __m512i sl = _mm512_add_epi64(yal, ybl), sh = _mm512_add_epi64(yah, ybh);
    sl = _mm512_add_epi64(sl, _mm512_shuffle_i64x2(sl, sl, 0x4E));
    sh = _mm512_add_epi64(sh, _mm512_shuffle_i64x2(sh, sh, 0x4E));
    A = v_combine(_mm512_add_epi64(yal, sl), _mm512_add_epi64(yah, sh));
    B = v_combine(_mm512_add_epi64(ybl, sl), _mm512_add_epi64(ybh, sh));
}
// sum of the 16 lanes of a and b (mod q): lane halves summed exactly
NEO_AVX512 static uint64_t v_hsum2(__m512i a, __m512i b) {
    const __m512i m32 = v_eps();
    const uint64_t sl = (uint64_t)_mm512_reduce_add_epi64(_mm512_add_epi64(_mm512_and_si512(a, m32), _mm512_and_si512(b, m32)));
    const uint64_t sh = (uint64_t)_mm512_reduce_add_epi64(_mm512_add_epi64(_mm512_srli_epi64(a, 32), _mm512_srli_epi64(b, 32)));
    const uint64_t hi = sh >> 32, lo = sh & GL_EPS;
    return add_carry_fix(sl + ((hi << 32) - hi), lo << 32);
}
// sum of the 8 lanes of a (mod q)
NEO_AVX512 static uint64_t v_hsum1(__m512i a) {
    const __m512i m32 = v_eps();
    const uint64_t sl = (uint64_t)_mm512_reduce_add_epi64(_mm512_and_si512(a, m32));
    const uint64_t sh = (uint64_t)_mm512_reduce_add_epi64(_mm512_srli_epi64(a, 32));
    const uint64_t hi = sh >> 32, lo = sh & GL_EPS;
    return add_carry_fix(sl + ((hi << 32) - hi), lo << 32);
}
NEO_AVX512 static void v_full16(__m512i& A, __m512i& B, const uint64_t* rc) {
    const __m512i xa = v_add_small(A, _mm512_loadu_si512(rc)), xb = v_add_small(B, _mm512_loadu_si512(rc + 8));
    const __m512i xa2 = v_mul(xa, xa), xb2 = v_mul(xb, xb);
    A = v_mul(v_mul(xa2, xa), v_mul(xa2, xa2));
    B = v_mul(v_mul(xb2, xb), v_mul(xb2, xb2));
    v_external16(A, B);
}
__attribute__((target("avx512f,bmi2"), noinline)) static void permute16_avx512(const Poseidon2<16>& P, uint64_t* st_io) {
    __m512i A = _mm512_loadu_si512(st_io), B = _mm512_loadu_si512(st_io + 8);
    v_external16(A, B);
    for (int r = 0; r < 4; r++) v_full16(A, B, P.rc_ext[r]);
    const __m512i muA = _mm512_maskz_loadu_epi64(0xFE, P.mu), muB = _mm512_loadu_si512(P.mu + 8);
    const __m512i muA_hi = _mm512_srli_epi64(muA, 32), muB_hi = _mm512_srli_epi64(muB, 32);
    uint64_t x0 = addq((uint64_t)_mm_cvtsi128_si64(_mm512_castsi512_si128(A)), P.rc_int[0]);
    __m512i va = _mm512_maskz_mov_epi64(0xFE, A), vb = B;
    uint64_t rest = v_hsum2(va, vb);
    const uint64_t mu0p1 = P.mu[0] + 1;
    for (int r = 0; r < 22; r++) {
        const __m512i pa = v_mul(va, muA, muA_hi), pb = v_mul(vb, muB, muB_hi);
        const uint64_t psum = v_hsum2(pa, pb);
        const uint64_t x = sbox7(x0);
        const uint64_t sum = canonq(red_small((u128)x + rest));
        const u128 addend = (u128)rest + (r + 1 < 22 ? P.rc_int[r + 1] : 0);
        x0 = red128((u128)mu0p1 * x + addend);
        const __m512i bs = _mm512_set1_epi64((long long)sum);
        va = v_add_small(pa, bs);
        vb = v_add_small(pb, bs);
        rest = red_small((u128)psum + red_small((u128)sum * 15));
    }
    A = _mm512_mask_set1_epi64(va, 0x01, (long long)x0);
    B = vb;
    for (int r = 4; r < 8; r++) v_full16(A, B, P.rc_ext[r]);
    const __m512i q = _mm512_set1_epi64((long long)GL_Q);
    A = _mm512_mask_sub_epi64(A, _mm512_cmpge_epu64_mask(A, q), A, q);
    B = _mm512_mask_sub_epi64(B, _mm512_cmpge_epu64_mask(B, q), B, q);
    _mm512_storeu_si512(st_io, A);
    _mm512_storeu_si512(st_io + 8, B);
}
// width 8: scalar full rounds; in the partial rounds lanes 1..7 in one vector
// (lane 0 masked to zero), whose products mu_i x_i do not wait for lane 0's
// S-box, so only that chain is serial (the scalar partial round is bound by
// the throughput of the seven scalar lane updates instead).  Bit-identical to
// permute_impl<8>.
__attribute__((target("avx512f,bmi2"), noinline)) static void permute8_avx512(const Poseidon2<8>& P, uint64_t* st_io) {
    uint64_t st[8];
#pragma GCC unroll 8
    for (int i = 0; i < 8; i++) st[i] = st_io[i];
    external_layer<8>(st);
    for (int r = 0; r < 4; r++) full_round<8>(st, P.rc_ext[r]);
    const __m512i mu = _mm512_maskz_loadu_epi64(0xFE, P.mu), mu_hi = _mm512_srli_epi64(mu, 32);
    __m512i v = _mm512_maskz_loadu_epi64(0xFE, st);
    uint64_t rest = v_hsum1(v);
    uint64_t x0 = addq(st[0], P.rc_int[0]);
    const uint64_t mu0p1 = P.mu[0] + 1;
    for (int r = 0; r < 22; r++) {
        const __m512i p = v_mul(v, mu, mu_hi);
        const uint64_t psum = v_hsum1(p);
        const uint64_t x = sbox7(x0);
        const uint64_t sum = canonq(red_small((u128)x + rest));
        const u128 addend = (u128)rest + (r + 1 < 22 ? P.rc_int[r + 1] : 0);
        x0 = red128((u128)mu0p1 * x + addend);
        v = _mm512_maskz_mov_epi64(0xFE, v_add_small(p, _mm512_set1_epi64((long long)sum)));
        rest = red_small((u128)psum + red_small((u128)sum * 7));
    }
    _mm512_storeu_si512(st, v);
    st[0] = x0;
    for (int r = 4; r < 8; r++) full_round<8>(st, P.rc_ext[r]);
#pragma GCC unroll 8
    for (int i = 0; i < 8; i++) st_io[i] = canonq(st[i]);
}
#undef NEO_AVX512

// AVX-512F (with BMI2) when the host has it, unless NEO_TRANSCRIPT_SCALAR is
// set (tests compare both paths)
static bool use_avx512() {
    static const bool on = [] {
        __builtin_cpu_init();
        return __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("bmi2") && !getenv("NEO_TRANSCRIPT_SCALAR");
    }();
    return on;
}
#endif

template <int W>
void Poseidon2<W>::permute(uint64_t* st_io) const {
#if defined(__x86_64__)
    if (use_avx512()) {
        if constexpr (W == 16)
            permute16_avx512(*this, st_io);
        else
            permute8_avx512(*this, st_io);
        return;
    }
#endif
    permute_impl<W>(*this, st_io);
}

template struct Poseidon2<8>;
template struct Poseidon2<16>;

// -------------------------------------------------------------- transcript --
static const char* APP_DOMAIN = "neo/transcript/v1|poseidon2-goldilocks-w8-r4";

Transcript::Transcript(const std::string& app_label) {
    memset(st_, 0, sizeof st_);
    append_message(APP_DOMAIN, reinterpret_cast<const uint8_t*>(app_label.data()), app_label.size());
}

void Transcript::permute() {
    transcript_perm().permute(st_);
    absorbed_ = 0;
    perms_++;
}

void Transcript::absorb_elem(uint64_t x) {
    if (absorbed_ >= RATE) permute();
    st_[absorbed_++] = x;
}

void Transcript::absorb_slice(const uint64_t* xs, size_t len) {
    size_t src = 0;
    while (absorbed_ < RATE && src < len) st_[absorbed_++] = xs[src++];
    if (absorbed_ == RATE) permute();
    while (len - src >= (size_t)RATE) {
        for (int i = 0; i < RATE; i++) st_[i] = xs[src + i];
        permute();
        src += RATE;
    }
    while (src < len) st_[absorbed_++] = xs[src++];
}

void Transcript::absorb_label(const std::string& label) {
    for (unsigned char c : label) absorb_elem((uint64_t)c);
}

void Transcript::append_message(const std::string& label, const uint8_t* msg, size_t len) {
    absorb_label(label);
    absorb_elem((uint64_t)len);
    for (size_t i = 0; i < len; i++) absorb_elem((uint64_t)msg[i]);
}

void Transcript::append_fields(const std::string& label, const uint64_t* fs, size_t n) {
    absorb_label(label);
    absorb_elem((uint64_t)n);
    absorb_slice(fs, n);
}

void Transcript::append_u64s(const std::string& label, const uint64_t* us, size_t n) {
    absorb_label(label);
    absorb_elem((uint64_t)n);
    for (size_t i = 0; i < n; i++) absorb_elem(gl::canon(us[i]));
}

uint64_t Transcript::challenge_field(const std::string& label) {
    append_message("chal/label", reinterpret_cast<const uint8_t*>(label.data()), label.size());
    absorb_elem(1);
    permute();
    return st_[0];
}

void Transcript::challenge_fields(const std::string& label, size_t n, uint64_t* out) {
    append_message("chal/label", reinterpret_cast<const uint8_t*>(label.data()), label.size());
    size_t got = 0;
    while (got < n) {
        absorb_elem(1);
        permute();
        for (int i = 0; i < 4 && got < n; i++) out[got++] = st_[i];
    }
}

void Transcript::digest32(uint8_t out[32]) {
    absorb_elem(1);
    permute();
    for (int i = 0; i < 4; i++)
        for (int b = 0; b < 8; b++) out[8 * i + b] = (uint8_t)(st_[i] >> (8 * b));
}

}  // namespace neo
