// ccs_fast.cuh -- Pi_CCS row rounds for ternary witness digits (b = 2).
//
// Included by ccs_oracle.cu inside its anonymous namespace (uses K, FTerms,
// MAX_DEG, ld_k, st_k, shfl_xor_k from there).
//
// The round polynomial of row round j (oracle.rs:416-503, 1047-1178) is
//   p_j(X) = sum_t eq_t(X) (f_t(X) + sum_q wg_q N(y_{q,t}(X))) + gamma^k eq_rin_t(X) eval_t(X)
// with N(y) = y^3 - y.  The beta_r equality table is a product over row bits,
// so after binding r_0..r_{j-1},
//   eq_t(X) = C_j eq(beta_j, X) E_j(t),  C_j = prod_{i<j} eq(beta_i, r_i),
//   E_j(t) = chi_{beta_{j+1..}}(t),
// and the kernels accumulate S(X) = sum_t E_j(t) (f_t(X) + NC_t(X)) and
// V(X) = sum_t eq_rin_t(X) eval_t(X); one reduction applies C_j eq(beta_j, X)
// and gamma^k (every quantity is exact in F_q, so the regrouping changes no bit).
//
// Rounds 0..2 (histogram of 8-row digit patterns).  With ternary digits, y of
// row round j <= 2 is a K-linear form in the 8 digits of the aligned 8-row
// block t8 that holds the pair, so
//   sum_t E_j(t) sum_q wg_q N(y_{q,t}) = sum_P H[P] F_j(P, X),
//   H[P] = sum_{(q,t8): pattern(q,t8) = P} E_2(t8) wg_q,
// where F_j(P, X) = sum_s chi_{beta_{j+1..2}}(s) N(y_{P,s}(X)) runs over the
// 2^(2-j) pairs s of the block.  N is odd and y is linear in the digits, so a
// pattern and its negation share one entry (the negated one enters with -w):
// 3280 entries.  H does not depend on any row challenge: round 0 builds it in
// one pass over the digits and rounds 0, 1, 2 each evaluate 3280 F_j's.
//
// Rounds 3 and 4 stream the digits (16- and 32-row blocks) and form
// y = sum_b chi_{r_<j}(b) z_b by 4-digit lookup tables (81 entries, one per
// base-3 digit group); round 4 writes the K table, rounds 5.. fold it.  The
// weighted N coefficients of every (pair, q) are summed unreduced (KAcc).

constexpr int NPAT = 3280;      // canonical nonzero 8-trit patterns
constexpr int HIST_LIMBS = 8;   // 16-bit limbs of a K value (re: 4, im: 4)
constexpr int HIST_T = 256;     // threads per histogram block
constexpr int HIST_MAX_Q = 256; // q per histogram block: <= 65536 items, so 16-bit limbs fit a u32 counter
constexpr int REC = MAX_DEG + 3;  // partial record: S coefficients [0, MAX_DEG), V coefficients [MAX_DEG, +3)
constexpr int FR = 256;           // threads per fast-row block
constexpr uint32_t P4W = 0x1B090301u;  // base-3 weights 1, 3, 9, 27 for __dp4a

// Out-of-line K products for code that runs once or a few times per warp
// (serial roles, late rounds): every call site shares one copy of the
// multiplication, so the instruction cache holds it; the hot streaming rounds
// keep the inlined form (C = false).
__device__ __noinline__ K kmul_n(K a, K b) { return gl::kmul(a, b); }
__device__ __noinline__ K ksqr_n(K a) { return gl::ksqr(a); }
template <bool C>
__device__ __forceinline__ K kmul_c(K a, K b) {
    if constexpr (C) return kmul_n(a, b);
    else return gl::kmul(a, b);
}
template <bool C>
__device__ __forceinline__ K ksqr_c(K a) {
    if constexpr (C) return ksqr_n(a);
    else return gl::ksqr(a);
}
template <bool C>
__device__ __forceinline__ K klerp_c(K a, K b, K r) { return gl::kadd(a, kmul_c<C>(gl::ksub(b, a), r)); }

// base-3 index of four ternary digits (bytes -1, 0, 1) and whether all four are ternary
__device__ __forceinline__ uint32_t p4_index(uint32_t x) { return __dp4a(__vadd4(x, 0x01010101u), P4W, 0u); }
__device__ __forceinline__ bool p4_ternary(uint32_t x) { return __vcmpgtu4(__vadd4(x, 0x01010101u), 0x02020202u) == 0; }

__global__ void ternary_check_kernel(const uint4* __restrict__ z, uint64_t n16, const uint8_t* __restrict__ tail,
                                     uint32_t ntail, uint32_t* __restrict__ bad) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    bool ok = true;
    for (; i < n16; i += stride) {
        uint4 v = z[i];
        ok &= p4_ternary(v.x) & p4_ternary(v.y) & p4_ternary(v.z) & p4_ternary(v.w);
    }
    if (blockIdx.x == 0 && threadIdx.x < ntail) {
        uint8_t b = tail[threadIdx.x];
        ok &= b == 0 || b == 1 || b == 0xFF;
    }
    if (!ok) atomicOr(bad, 1u);
}

struct HistArgs {
    const int8_t* Z;   // [nq][m]
    uint64_t m;
    uint32_t nq;
    uint32_t n_t8;     // m / 8
    uint32_t q_chunk;  // q per block (<= HIST_MAX_Q)
    const K* wg;       // [nq]
    const K* Ew;       // split: E_3 [n_t8 / 2] (weight of block t8 is Ew[t8 >> 1]); else E_2 [n_t8]
    int split;         // blockIdx.z = parity of t8: one histogram per parity
    uint32_t* partial; // [gridDim.z][gridDim.y][gridDim.x][HIST_LIMBS][NPAT]
};

// One thread per 8-row block t8, a range of q per block.  Each nonzero
// (q, t8) adds +-w(t8) wg_q to its pattern's counters: eight 16-bit limbs
// (re: 0..3, im: 4..7) in u32 shared-memory counters, at most 65536 adds per
// block so no counter overflows.  The counters are limb-major, so the lanes
// of a warp (random patterns) spread over the banks.  Split: the even and the
// odd 8-row blocks (the lo and hi halves of the 16-row blocks of round 3)
// fill separate histograms, weighted by E_3 of their 16-row block.
__global__ void __launch_bounds__(HIST_T) ccs_hist_kernel(const HistArgs a) {
    extern __shared__ uint32_t s_hist[];  // [HIST_LIMBS][NPAT], then wg of the block's q range
    K* s_wg = reinterpret_cast<K*>(s_hist + NPAT * HIST_LIMBS);
    const int tid = threadIdx.x;
    for (int i = tid; i < NPAT * HIST_LIMBS; i += HIST_T) s_hist[i] = 0;
    const uint32_t q0 = blockIdx.y * a.q_chunk;
    const uint32_t q1 = min(a.nq, q0 + a.q_chunk);
    for (uint32_t q = q0 + tid; q < q1; q += HIST_T) s_wg[q - q0] = a.wg[q];
    __syncthreads();
    const uint32_t u = blockIdx.x * HIST_T + tid;
    const uint32_t t8 = a.split ? 2 * u + blockIdx.z : u;
    if (t8 < a.n_t8) {
        const K e = a.Ew[a.split ? (t8 >> 1) : t8];
        const int8_t* zp = a.Z + (uint64_t)q0 * a.m + 8ull * t8;
        constexpr int BATCH = 8;  // loads in flight per thread
        for (uint32_t qb = q0; qb < q1; qb += BATCH) {
          uint2 vb[BATCH];
#pragma unroll
          for (int i = 0; i < BATCH; i++)
              vb[i] = qb + i < q1 ? __ldg(reinterpret_cast<const uint2*>(zp + (uint64_t)(qb - q0 + i) * a.m))
                                 : make_uint2(0, 0);
#pragma unroll
          for (int i = 0; i < BATCH; i++) {
            const uint2 v = vb[i];
            const uint32_t q = qb + i;
            if ((v.x | v.y) == 0) continue;
            const int P = (int)(p4_index(v.x) + 81u * p4_index(v.y));
            K w = gl::kmul(e, s_wg[q - q0]);
            int idx;
            if (P > NPAT) {
                idx = P - (NPAT + 1);
            } else {
                idx = NPAT - 1 - P;  // the negated pattern 6560 - P
                w = gl::kneg(w);
            }
#pragma unroll
            for (int l = 0; l < 4; l++) {
                atomicAdd(s_hist + l * NPAT + idx, (uint32_t)((w.re >> (16 * l)) & 0xFFFF));
                atomicAdd(s_hist + (4 + l) * NPAT + idx, (uint32_t)((w.im >> (16 * l)) & 0xFFFF));
            }
          }
        }
    }
    __syncthreads();
    uint32_t* out = a.partial +
                    (((uint64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * (NPAT * HIST_LIMBS);
    for (int i = tid; i < NPAT * HIST_LIMBS / 4; i += HIST_T)
        reinterpret_cast<uint4*>(out)[i] = reinterpret_cast<const uint4*>(s_hist)[i];
}

// H64[z][l][p] += the block counters of one slice of the blocks of histogram
// z; one thread per counter, consecutive threads on consecutive counters.
// Each sum stays below 2^52 (2^20 blocks of counters < 2^32).
constexpr int HIST_SUM_SLICE = 8;
__global__ void __launch_bounds__(256) ccs_hist_sum_kernel(const uint32_t* __restrict__ partial, uint32_t nblk,
                                                           unsigned long long* __restrict__ H64) {
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i >= NPAT * HIST_LIMBS) return;
    const uint32_t z = blockIdx.z;
    const uint32_t b0 = blockIdx.y * HIST_SUM_SLICE, b1 = min(nblk, b0 + HIST_SUM_SLICE);
    const uint32_t* src = partial + (uint64_t)z * nblk * NPAT * HIST_LIMBS + i;
    uint64_t acc = 0;
    for (uint32_t b = b0; b < b1; b++) acc += __ldg(src + (uint64_t)b * NPAT * HIST_LIMBS);
    if (acc) atomicAdd(H64 + (uint64_t)z * NPAT * HIST_LIMBS + i, (unsigned long long)acc);
}

// H[p] from its eight limb sums (limb l has weight 2^(16 l); 2^0 .. 2^48 are canonical)
__device__ __forceinline__ K hist_value(const unsigned long long* H64, int p) {
    uint64_t re = 0, im = 0;  // H64 points at one histogram [HIST_LIMBS][NPAT]
#pragma unroll
    for (int l = 0; l < 4; l++) {
        const uint64_t pw = 1ull << (16 * l);
        re = gl::add(re, gl::mul(gl::canon(H64[l * NPAT + p]), pw));
        im = gl::add(im, gl::mul(gl::canon(H64[(4 + l) * NPAT + p]), pw));
    }
    return gl::kmk(re, im);
}

// coefficients of N(lo + (hi - lo) X) = c0 + c1 X + c2 X^2 + c3 X^3
template <bool C = false>
__device__ __forceinline__ void n_coeffs(K lo, K hi, K c[4]) {
    const K b = gl::ksub(hi, lo);
    const K a2 = ksqr_c<C>(lo), b2 = ksqr_c<C>(b);
    const K a2b = kmul_c<C>(a2, b), ab2 = kmul_c<C>(lo, b2);
    c[0] = gl::ksub(kmul_c<C>(a2, lo), lo);
    c[1] = gl::ksub(gl::kadd(gl::kdbl(a2b), a2b), b);
    c[2] = gl::kadd(gl::kdbl(ab2), ab2);
    c[3] = kmul_c<C>(b2, b);
}

__device__ __forceinline__ K eq_lin(K a, K b) {  // (1 - a)(1 - b) + a b
    return gl::kadd(kmul_n(gl::ksub(gl::kone(), a), gl::ksub(gl::kone(), b)), kmul_n(a, b));
}

// chi_{pts[0..n)}(b)
__device__ __forceinline__ K chi_of(const K* pts, int n, uint32_t b) {
    K w = gl::kone();
    for (int i = 0; i < n; i++) w = kmul_n(w, ((b >> i) & 1) ? pts[i] : gl::ksub(gl::kone(), pts[i]));
    return w;
}

// block sum of v[0..n) into rec[0..n), zeros in rec[n..REC); n <= REC
__device__ __forceinline__ void block_sum_rec(const K* v, int n, K* rec) {
    __shared__ K s_red[FR / 32][REC];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll 1
    for (int d = 0; d < n; d++) {
        K x = v[d];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = gl::kadd(x, shfl_xor_k(x, o));
        if (lane == 0) s_red[warp][d] = x;
    }
    __syncthreads();
    if (threadIdx.x < REC) {
        K x = gl::kzero();
        if ((int)threadIdx.x < n)
            for (int w = 0; w < FR / 32; w++) x = gl::kadd(x, s_red[w][threadIdx.x]);
        st_k(rec + threadIdx.x, x);
    }
}

// One row round is one launch of ccs_fast_round_kernel: its blocks take one
// of three roles, in this order, and each writes one partial record:
//   moment blocks (rounds 0..2): sum_P H[P] F_j(P, X), one thread per pattern;
//   small-table blocks: fold the f-variable / eq_rin / eval tables, add
//     E_j(t) f_t(X) to S and eq_rin_t(X) eval_t(X) to V, one thread per pair;
//   NC blocks (rounds >= 3): E_j(t) sum_q wg_q N(y_{q,t}(X)) over a q chunk,
//     one thread per (pair, chunk).
// The last block to finish (an atomic ticket) sums the records and writes the
// round's coefficients C_j eq(beta_j, X) S(X) + gamma^k V(X).
struct FastRoundArgs {
    int j;
    uint32_t n_mom, n_small;     // blocks of the first two roles; the rest are NC blocks
    // moments
    const unsigned long long* H64;  // [1 + split][HIST_LIMBS][NPAT]
    int split;                   // H64 holds the even / odd 8-row-block histograms (weights E_3)
    K beta1, beta2, beta3;       // beta_r[1..3] (beta3 only with split)
    // small tables: f variables at slots 1..n_fvar, eq_rin / eval at idx_eqrin / idx_eval
    const K* small_in;
    K* small_out;
    uint64_t small_len_in, small_len_out;
    int fold;
    K r;                         // r_{j-1}
    int n_small_tab;
    int idx_eqrin, idx_eval;
    FTerms f;
    int fdeg;                    // degree of f (<= MAX_DEG - 1)
    const K* E;                  // E_j [pairs]
    uint64_t pairs;
    // NC
    const K* chals;              // device r_0..r_{j-1}
    const int8_t* Z;             // [nq][m]
    uint64_t m;
    const K* nc_in;              // T_{j-1} [nq][nc_len_in] (rounds >= 5)
    uint64_t nc_len_in;
    K* nc_out;                   // T_j [nq][nc_len_out] (rounds 4.., null in the last round)
    uint64_t nc_len_out;
    const K* wg;                 // [nq]
    uint32_t nq, q_chunk, n_chunk;
    // reduction
    K* partials;                 // [gridDim.x][REC]
    unsigned int* ticket;        // zero between launches (atomicInc wraps it)
    int ncoef;
    K beta[32];                  // beta_r
    K gamma_to_k;
    K* Cs;                       // [ell]: C_j of each round (written by round j)
    K* coeffs_out;               // [ncoef]
};

// The roles and the final reduction run as out-of-line functions with rolled
// loops: a launch of a late round has few warps, and long straight-line
// K-multiplication code there stalls on instruction fetch.
__device__ __noinline__ void mom_role(const FastRoundArgs& a, uint32_t blk, K* rec) {
    K c[4] = {gl::kzero(), gl::kzero(), gl::kzero(), gl::kzero()};
    const int p = blk * FR + threadIdx.x;
    if (p < NPAT) {
        // split: an 8-row block of parity z weighs E_2(t8) = eq(beta_3, z) E_3(t8 >> 1)
        const K h = a.split ? gl::kadd(kmul_n(gl::ksub(gl::kone(), a.beta3), hist_value(a.H64, p)),
                                       kmul_n(a.beta3, hist_value(a.H64 + NPAT * HIST_LIMBS, p)))
                            : hist_value(a.H64, p);
        if (!gl::kiszero(h)) {
            int tr[8];
            int P = p + NPAT + 1;
#pragma unroll
            for (int i = 0; i < 8; i++) { tr[i] = P % 3 - 1; P /= 3; }
            K F[4] = {gl::kzero(), gl::kzero(), gl::kzero(), gl::kzero()};
            if (a.j == 0) {
                // pair s: lo = tr[2s], hi = tr[2s + 1] (small integers); weight chi_{beta1, beta2}(s)
#pragma unroll
                for (int s = 0; s < 4; s++) {
                    const int lo = tr[2 * s], b = tr[2 * s + 1] - lo;
                    const int n1 = b * (3 * lo * lo - 1), n2 = 3 * lo * b * b, n3 = b * b * b;
                    if (!(n1 | n2 | n3)) continue;
                    const K ws = kmul_n((s & 1) ? a.beta1 : gl::ksub(gl::kone(), a.beta1),
                                          (s & 2) ? a.beta2 : gl::ksub(gl::kone(), a.beta2));
                    F[1] = gl::kadd(F[1], gl::kscale_small(ws, n1));
                    F[2] = gl::kadd(F[2], gl::kscale_small(ws, n2));
                    F[3] = gl::kadd(F[3], gl::kscale_small(ws, n3));
                }
            } else {
                const int j = a.j, half = 1 << j, nsub = 1 << (2 - j);
                K w[4];
                for (int b = 0; b < half; b++) w[b] = chi_of(a.chals, j, b);
                for (int s = 0; s < nsub; s++) {
                    K lo = gl::kzero(), hi = gl::kzero();
                    for (int b = 0; b < half; b++) {
                        const int dl = tr[2 * half * s + b], dh = tr[2 * half * s + half + b];
                        if (dl) lo = dl > 0 ? gl::kadd(lo, w[b]) : gl::ksub(lo, w[b]);
                        if (dh) hi = dh > 0 ? gl::kadd(hi, w[b]) : gl::ksub(hi, w[b]);
                    }
                    K n[4];
                    n_coeffs<true>(lo, hi, n);
                    if (j == 1) {
                        const K ws = s ? a.beta2 : gl::ksub(gl::kone(), a.beta2);
                        for (int d = 0; d < 4; d++) F[d] = gl::kadd(F[d], kmul_n(ws, n[d]));
                    } else {
                        for (int d = 0; d < 4; d++) F[d] = n[d];
                    }
                }
            }
            for (int d = 0; d < 4; d++) c[d] = kmul_n(h, F[d]);
        }
    }
    block_sum_rec(c, 4, rec);
}

__device__ __noinline__ void small_role(const FastRoundArgs& a, uint32_t blk, K* rec) {
    K out[REC];
#pragma unroll
    for (int d = 0; d < REC; d++) out[d] = gl::kzero();
    const uint64_t t = blk * (uint64_t)FR + threadIdx.x;
    if (t < a.pairs) {
        K lo_s[2 + MAX_FVAR + 2], hi_s[2 + MAX_FVAR + 2];
#pragma unroll
        for (int s = 1; s < 2 + MAX_FVAR + 2; s++) {
            if (s >= a.n_small_tab) break;
            K lo, hi;
            if (a.fold) {
                const K* in = a.small_in + (uint64_t)s * a.small_len_in + 4 * t;
                lo = klerp_c<true>(ld_k(in), ld_k(in + 1), a.r);
                hi = klerp_c<true>(ld_k(in + 2), ld_k(in + 3), a.r);
                if (a.small_out) {
                    K* o = a.small_out + (uint64_t)s * a.small_len_out + 2 * t;
                    st_k(o, lo);
                    st_k(o + 1, hi);
                }
            } else {
                const K* in = a.small_in + (uint64_t)s * a.small_len_in + 2 * t;
                lo = ld_k(in);
                hi = ld_k(in + 1);
            }
            lo_s[s] = lo;
            hi_s[s] = hi;
        }
        // f_t(X) = sum_terms coeff prod_v (a_v + b_v X)^exp, degree <= fdeg
        K S[MAX_DEG], tp[MAX_DEG];
#pragma unroll 1
        for (int d = 0; d < MAX_DEG; d++) S[d] = gl::kzero();
#pragma unroll 1
        for (int tt = 0; tt < a.f.n_terms; tt++) {
#pragma unroll 1
            for (int d = 0; d < MAX_DEG; d++) tp[d] = gl::kzero();
            tp[0] = a.f.coeff[tt];
            int deg = 0;  // degree of tp so far
#pragma unroll 1
            for (int vv = 0; vv < a.f.n_vars[tt]; vv++) {
                const int pos = a.f.var_pos[tt][vv];
                const K av = lo_s[1 + pos], bv = gl::ksub(hi_s[1 + pos], av);
#pragma unroll 1
                for (int e = 0; e < a.f.var_exp[tt][vv] && deg < a.fdeg; e++) {
                    deg++;
                    tp[deg] = kmul_n(bv, tp[deg - 1]);
#pragma unroll 1
                    for (int d = deg - 1; d >= 1; d--) tp[d] = gl::kadd(kmul_n(av, tp[d]), kmul_n(bv, tp[d - 1]));
                    tp[0] = kmul_n(av, tp[0]);
                }
            }
#pragma unroll 1
            for (int d = 0; d <= deg; d++) S[d] = gl::kadd(S[d], tp[d]);
        }
        const K e = a.E[t];
#pragma unroll 1
        for (int d = 0; d <= a.fdeg; d++) S[d] = kmul_n(e, S[d]);
#pragma unroll
        for (int d = 0; d < MAX_DEG; d++) out[d] = d <= a.fdeg ? S[d] : gl::kzero();
        if (a.idx_eval >= 0) {
            const K r0 = lo_s[a.idx_eqrin], r1 = gl::ksub(hi_s[a.idx_eqrin], r0);
            const K v0 = lo_s[a.idx_eval], v1 = gl::ksub(hi_s[a.idx_eval], v0);
            out[MAX_DEG] = kmul_n(r0, v0);
            out[MAX_DEG + 1] = gl::kadd(kmul_n(r0, v1), kmul_n(r1, v0));
            out[MAX_DEG + 2] = kmul_n(r1, v1);
        }
    }
    block_sum_rec(out, REC, rec);
}

// Round 3, separable part.  With lo, hi the K-linear forms of the even and
// odd 8-row blocks of a 16-row block, N(lo + (hi - lo) X) has coefficients
//   c0 = lo^3 - lo,                 c1 = 3 lo^2 hi - 3 lo^3 - hi + lo,
//   c2 = 3 lo hi^2 - 6 lo^2 hi + 3 lo^3,   c3 = hi^3 - 3 lo hi^2 + 3 lo^2 hi - lo^3.
// The terms in lo or hi alone are odd functions of one 8-row pattern, so they
// come from the split histograms: SA_k = sum_P H_even[P] LV(P)^k and SB_k
// with H_odd (LV(P) = sum_b chi_{r_0..r_2}(b) trit_b(P), E_3 already in H).
// The NC blocks of round 3 add the cross terms lo^2 hi and lo hi^2.
__device__ __noinline__ void sep_role(const FastRoundArgs& a, uint32_t blk, K* rec) {
    __shared__ K s_w8[8];
    if (threadIdx.x < 8) s_w8[threadIdx.x] = chi_of(a.chals, 3, threadIdx.x);
    __syncthreads();
    K c[4] = {gl::kzero(), gl::kzero(), gl::kzero(), gl::kzero()};
    const int p = blk * FR + threadIdx.x;
    if (p < NPAT) {
        const K hA = hist_value(a.H64, p), hB = hist_value(a.H64 + NPAT * HIST_LIMBS, p);
        if (!gl::kiszero(hA) || !gl::kiszero(hB)) {
            int P = p + NPAT + 1;
            K lv = gl::kzero();
#pragma unroll 1
            for (int i = 0; i < 8; i++) {
                const int d = P % 3 - 1;
                P /= 3;
                if (d) lv = d > 0 ? gl::kadd(lv, s_w8[i]) : gl::ksub(lv, s_w8[i]);
            }
            const K l3 = kmul_n(ksqr_n(lv), lv);
            const K sa1 = kmul_n(hA, lv), sa3 = kmul_n(hA, l3), sb1 = kmul_n(hB, lv), sb3 = kmul_n(hB, l3);
            const K sa3x3 = gl::kadd(gl::kdbl(sa3), sa3);
            c[0] = gl::ksub(sa3, sa1);
            c[1] = gl::ksub(gl::ksub(sa1, sa3x3), sb1);
            c[2] = sa3x3;
            c[3] = gl::ksub(sb3, sa3);
        }
    }
    block_sum_rec(c, 4, rec);
}

template <int MODE, bool C>
__device__ __forceinline__ void nc_role(const FastRoundArgs& a, uint32_t blk, K* rec, K* s_wg) {
    constexpr int NLUT = MODE == 3 ? 2 : (MODE == 4 ? 4 : 0);
    __shared__ K s_lut[NLUT ? NLUT * 81 : 1];
    __shared__ K s_w[16];
    const uint64_t gid = blk * (uint64_t)FR + threadIdx.x;
    const bool live = gid < a.pairs * a.n_chunk;
    const uint64_t t = live ? gid % a.pairs : 0;
    const uint32_t c = live ? (uint32_t)(gid / a.pairs) : 0;
    if constexpr (NLUT > 0) {
        if (threadIdx.x < (1u << a.j)) s_w[threadIdx.x] = chi_of(a.chals, a.j, threadIdx.x);
        __syncthreads();
        for (int e = threadIdx.x; e < NLUT * 81; e += FR) {
            const int g = e / 81;
            int P = e % 81;
            K v = gl::kzero();
            for (int i = 0; i < 4; i++) {
                const int d = P % 3 - 1;
                P /= 3;
                if (d) v = d > 0 ? gl::kadd(v, s_w[4 * g + i]) : gl::ksub(v, s_w[4 * g + i]);
            }
            s_lut[e] = v;
        }
    }
    for (uint32_t q = threadIdx.x; q < a.nq; q += FR) s_wg[q] = a.wg[q];
    __syncthreads();

    K out[4] = {gl::kzero(), gl::kzero(), gl::kzero(), gl::kzero()};
    if (live) {
        constexpr int NACC = MODE == 3 ? 2 : 4;
        gl::KAcc acc[NACC];
#pragma unroll
        for (int d = 0; d < NACC; d++) gl::kacc_zero(acc[d]);
        const uint32_t q0 = c * a.q_chunk, q1 = min(a.nq, q0 + a.q_chunk);
        // the next q's inputs are loaded before the current one is evaluated
        uint4 nv = make_uint4(0, 0, 0, 0), nu = make_uint4(0, 0, 0, 0);
        ulonglong2 nx[4];
        auto fetch = [&](uint32_t q) {
            if (q >= q1) return;
            if constexpr (MODE == 3) {
                nv = __ldg(reinterpret_cast<const uint4*>(a.Z + (uint64_t)q * a.m + 16 * t));
            } else if constexpr (MODE == 4) {
                const uint4* zp = reinterpret_cast<const uint4*>(a.Z + (uint64_t)q * a.m + 32 * t);
                nv = __ldg(zp);
                nu = __ldg(zp + 1);
            } else {
                const ulonglong2* in = reinterpret_cast<const ulonglong2*>(a.nc_in + (uint64_t)q * a.nc_len_in + 4 * t);
#pragma unroll
                for (int i = 0; i < 4; i++) nx[i] = __ldg(in + i);
            }
        };
        fetch(q0);
        for (uint32_t q = q0; q < q1; q++) {
            const uint4 cv = nv, cu = nu;
            ulonglong2 cx[4];
#pragma unroll
            for (int i = 0; i < 4; i++) cx[i] = nx[i];
            fetch(q + 1);
            K lo, hi;
            if constexpr (MODE == 3) {
                const uint4 v = cv;
                if ((v.x | v.y) == 0 || (v.z | v.w) == 0) continue;  // a zero half zeroes both cross terms
                lo = gl::kadd(s_lut[p4_index(v.x)], s_lut[81 + p4_index(v.y)]);
                hi = gl::kadd(s_lut[p4_index(v.z)], s_lut[81 + p4_index(v.w)]);
            } else if constexpr (MODE == 4) {
                const uint4 v = cv, u = cu;
                const bool zero = (v.x | v.y | v.z | v.w | u.x | u.y | u.z | u.w) == 0;
                if (zero) {
                    lo = hi = gl::kzero();
                } else {
                    lo = gl::kadd(gl::kadd(s_lut[p4_index(v.x)], s_lut[81 + p4_index(v.y)]),
                                  gl::kadd(s_lut[162 + p4_index(v.z)], s_lut[243 + p4_index(v.w)]));
                    hi = gl::kadd(gl::kadd(s_lut[p4_index(u.x)], s_lut[81 + p4_index(u.y)]),
                                  gl::kadd(s_lut[162 + p4_index(u.z)], s_lut[243 + p4_index(u.w)]));
                }
                if (a.nc_out) {
                    K* o = a.nc_out + (uint64_t)q * a.nc_len_out + 2 * t;
                    st_k(o, lo);
                    st_k(o + 1, hi);
                }
                if (zero) continue;
            } else {
                const K x0 = gl::kmk(cx[0].x, cx[0].y), x1 = gl::kmk(cx[1].x, cx[1].y);
                const K x2 = gl::kmk(cx[2].x, cx[2].y), x3 = gl::kmk(cx[3].x, cx[3].y);
                lo = klerp_c<C>(x0, x1, a.r);
                hi = klerp_c<C>(x2, x3, a.r);
                if (a.nc_out) {
                    K* o = a.nc_out + (uint64_t)q * a.nc_len_out + 2 * t;
                    st_k(o, lo);
                    st_k(o + 1, hi);
                }
                if (gl::kiszero(lo) && gl::kiszero(hi)) continue;
            }
            const K w = s_wg[q];
            const uint64_t w7 = gl::mul7(w.im);
            if constexpr (MODE == 3) {
                // cross terms only (the separable ones come from the split histograms)
                gl::kacc_mad(acc[0], w, w7, kmul_c<C>(ksqr_c<C>(lo), hi));
                gl::kacc_mad(acc[1], w, w7, kmul_c<C>(lo, ksqr_c<C>(hi)));
            } else {
                K n[4];
                n_coeffs<C>(lo, hi, n);
#pragma unroll
                for (int d = 0; d < 4; d++) gl::kacc_mad(acc[d], w, w7, n[d]);
            }
        }
        const K e = a.E[t];
        if constexpr (MODE == 3) {
            const K x21 = gl::kacc_reduce(acc[0]), x12 = gl::kacc_reduce(acc[1]);
            const K x21x3 = gl::kadd(gl::kdbl(x21), x21), x12x3 = gl::kadd(gl::kdbl(x12), x12);
            out[1] = kmul_c<C>(e, x21x3);
            out[2] = kmul_c<C>(e, gl::ksub(x12x3, gl::kdbl(x21x3)));
            out[3] = kmul_c<C>(e, gl::ksub(x21x3, x12x3));
        } else {
#pragma unroll
            for (int d = 0; d < 4; d++) out[d] = kmul_c<C>(e, gl::kacc_reduce(acc[d]));
        }
    }
    block_sum_rec(out, 4, rec);
}

// Sums the records of every block of the launch (run by the last block).
__device__ __noinline__ void round_final_reduce(const FastRoundArgs& a) {
    __shared__ K s_tot[FR / 32][REC];
    K s[REC];
#pragma unroll
    for (int d = 0; d < REC; d++) s[d] = gl::kzero();
    for (uint32_t r = threadIdx.x; r < gridDim.x; r += FR) {
        const ulonglong2* p = reinterpret_cast<const ulonglong2*>(a.partials + (uint64_t)r * REC);
#pragma unroll
        for (int d = 0; d < REC; d++) {
            const ulonglong2 v = __ldcg(p + d);
            s[d] = gl::kadd(s[d], gl::kmk(v.x, v.y));
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < REC; d++) {
        K x = s[d];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = gl::kadd(x, shfl_xor_k(x, o));
        if (lane == 0) s_tot[warp][d] = x;
    }
    __syncthreads();
    __shared__ K s_S[REC];
    if (threadIdx.x < REC) {
        K x = gl::kzero();
#pragma unroll 1
        for (int w = 0; w < FR / 32; w++) x = gl::kadd(x, s_tot[w][threadIdx.x]);
        s_S[threadIdx.x] = x;
    }
    __syncthreads();
    if (threadIdx.x < (unsigned)a.ncoef) {
        // C_j eq(beta_j, X) = e0 + e1 X; coefficient d = e0 S_d + e1 S_{d-1} + gamma^k V_d
        // C_j = C_{j-1} eq(beta_{j-1}, r_{j-1}), C_0 = 1; kept on the device per round
        const K Cj = a.j == 0 ? gl::kone() : kmul_n(ld_k(a.Cs + a.j - 1), eq_lin(a.beta[a.j - 1], a.chals[a.j - 1]));
        if (threadIdx.x == 0) st_k(a.Cs + a.j, Cj);
        const K bj = a.beta[a.j];
        const K e0 = kmul_n(Cj, gl::ksub(gl::kone(), bj));
        const K e1 = kmul_n(Cj, gl::ksub(gl::kdbl(bj), gl::kone()));
        const int d = threadIdx.x;
        K v = gl::kzero();
        if (d < MAX_DEG) v = kmul_n(e0, s_S[d]);
        if (d >= 1 && d - 1 < MAX_DEG) v = gl::kadd(v, kmul_n(e1, s_S[d - 1]));
        if (d < 3) v = gl::kadd(v, kmul_n(a.gamma_to_k, s_S[MAX_DEG + d]));
        st_k(a.coeffs_out + d, v);
    }
}

// MODE 0: rounds 0..2 (moment and small-table blocks); 3 / 4: stream 16- /
// 32-row digit blocks; 5: fold the K table.
template <int MODE, bool C>
__global__ void __launch_bounds__(FR, 2) ccs_fast_round_kernel(const __grid_constant__ FastRoundArgs a) {
    extern __shared__ K s_wg[];  // [nq] for NC blocks
    const uint32_t b = blockIdx.x;
    K* rec = a.partials + (uint64_t)b * REC;
    if (b < a.n_mom) {
        if constexpr (MODE == 3) sep_role(a, b, rec);
        else mom_role(a, b, rec);
    } else if (b < a.n_mom + a.n_small) {
        small_role(a, b - a.n_mom, rec);
    } else {
        if constexpr (MODE != 0) nc_role<MODE, C>(a, b - a.n_mom - a.n_small, rec, s_wg);
    }
    // the record is written by threads < REC; publish it, then take a ticket
    __threadfence();
    __syncthreads();
    __shared__ unsigned int s_last;
    if (threadIdx.x == 0) s_last = atomicInc(a.ticket, gridDim.x - 1) == gridDim.x - 1;
    __syncthreads();
    if (s_last) {
        __threadfence();
        round_final_reduce(a);
    }
}
