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
    const K* E8;       // E_2, [n_t8]
    uint32_t* partial; // [gridDim.y][gridDim.x][NPAT][HIST_LIMBS]
};

// One thread per 8-row block t8, a range of q per block.  Each nonzero
// (q, t8) adds +-E_2(t8) wg_q to its pattern's counters: eight 16-bit limbs
// in u32 shared-memory counters (at most 65536 adds per block).
__global__ void __launch_bounds__(HIST_T) ccs_hist_kernel(const HistArgs a) {
    extern __shared__ uint32_t s_hist[];  // [NPAT][HIST_LIMBS], then wg of the block's q range
    K* s_wg = reinterpret_cast<K*>(s_hist + NPAT * HIST_LIMBS);
    const int tid = threadIdx.x;
    for (int i = tid; i < NPAT * HIST_LIMBS; i += HIST_T) s_hist[i] = 0;
    const uint32_t q0 = blockIdx.y * a.q_chunk;
    const uint32_t q1 = min(a.nq, q0 + a.q_chunk);
    for (uint32_t q = q0 + tid; q < q1; q += HIST_T) s_wg[q - q0] = a.wg[q];
    __syncthreads();
    const uint32_t t8 = blockIdx.x * HIST_T + tid;
    if (t8 < a.n_t8) {
        const K e = a.E8[t8];
        const int8_t* zp = a.Z + (uint64_t)q0 * a.m + 8ull * t8;
        for (uint32_t q = q0; q < q1; q++, zp += a.m) {
            const uint2 v = *reinterpret_cast<const uint2*>(zp);
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
            uint32_t* h = s_hist + idx * HIST_LIMBS;
            atomicAdd(h + 0, (uint32_t)(w.re & 0xFFFF));
            atomicAdd(h + 1, (uint32_t)((w.re >> 16) & 0xFFFF));
            atomicAdd(h + 2, (uint32_t)((w.re >> 32) & 0xFFFF));
            atomicAdd(h + 3, (uint32_t)(w.re >> 48));
            atomicAdd(h + 4, (uint32_t)(w.im & 0xFFFF));
            atomicAdd(h + 5, (uint32_t)((w.im >> 16) & 0xFFFF));
            atomicAdd(h + 6, (uint32_t)((w.im >> 32) & 0xFFFF));
            atomicAdd(h + 7, (uint32_t)(w.im >> 48));
        }
    }
    __syncthreads();
    uint32_t* out = a.partial + ((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * (NPAT * HIST_LIMBS);
    for (int i = tid; i < NPAT * HIST_LIMBS / 4; i += HIST_T)
        reinterpret_cast<uint4*>(out)[i] = reinterpret_cast<const uint4*>(s_hist)[i];
}

// H[p] = sum over blocks of the limb counters, recombined mod q.  Block:
// 32 patterns x 8 limbs (one thread each), summing nblk counters in u64
// (each counter < 2^32; nblk <= 2^20 keeps the sum < 2^52).
__global__ void __launch_bounds__(256) ccs_hist_reduce_kernel(const uint32_t* __restrict__ partial, uint32_t nblk,
                                                              K* __restrict__ H) {
    __shared__ uint64_t s[32][HIST_LIMBS];
    const int tid = threadIdx.x;
    const uint32_t p = blockIdx.x * 32 + tid / HIST_LIMBS;
    const int l = tid % HIST_LIMBS;
    uint64_t acc = 0;
    if (p < NPAT) {
        const uint32_t* src = partial + (uint64_t)p * HIST_LIMBS + l;
        uint32_t b = 0;
        for (; b + 4 <= nblk; b += 4) {
            const uint64_t st = (uint64_t)NPAT * HIST_LIMBS;
            acc += (uint64_t)src[b * st] + src[(b + 1) * st] + src[(b + 2) * st] + src[(b + 3) * st];
        }
        for (; b < nblk; b++) acc += src[(uint64_t)b * NPAT * HIST_LIMBS];
    }
    s[tid / HIST_LIMBS][l] = acc;
    __syncthreads();
    if (tid < 32 && blockIdx.x * 32 + tid < NPAT) {
        // limb l has weight 2^(16 (l mod 4)); 2^0, 2^16, 2^32, 2^48 are canonical
        uint64_t re = 0, im = 0;
        for (int i = 0; i < 4; i++) {
            const uint64_t pw = 1ull << (16 * i);
            re = gl::add(re, gl::mul(gl::canon(s[tid][i]), pw));
            im = gl::add(im, gl::mul(gl::canon(s[tid][4 + i]), pw));
        }
        H[blockIdx.x * 32 + tid] = gl::kmk(re, im);
    }
}

// coefficients of N(lo + (hi - lo) X) = c0 + c1 X + c2 X^2 + c3 X^3
__device__ __forceinline__ void n_coeffs(K lo, K hi, K c[4]) {
    const K b = gl::ksub(hi, lo);
    const K a2 = gl::ksqr(lo), b2 = gl::ksqr(b);
    const K a2b = gl::kmul(a2, b), ab2 = gl::kmul(lo, b2);
    c[0] = gl::ksub(gl::kmul(a2, lo), lo);
    c[1] = gl::ksub(gl::kadd(gl::kdbl(a2b), a2b), b);
    c[2] = gl::kadd(gl::kdbl(ab2), ab2);
    c[3] = gl::kmul(b2, b);
}

__device__ __forceinline__ K eq_lin(K a, K b) {  // (1 - a)(1 - b) + a b
    return gl::kadd(gl::kmul(gl::ksub(gl::kone(), a), gl::ksub(gl::kone(), b)), gl::kmul(a, b));
}

// chi_{pts[0..n)}(b)
__device__ __forceinline__ K chi_of(const K* pts, int n, uint32_t b) {
    K w = gl::kone();
    for (int i = 0; i < n; i++) w = gl::kmul(w, ((b >> i) & 1) ? pts[i] : gl::ksub(gl::kone(), pts[i]));
    return w;
}

// block sum of v[0..n) into rec[0..n), zeros in rec[n..REC); n <= REC
__device__ __forceinline__ void block_sum_rec(K* v, int n, K* rec) {
    __shared__ K s_red[FR / 32][REC];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) x = gl::kadd(x, s_red[w][threadIdx.x]);
        rec[threadIdx.x] = x;
    }
}

struct MomArgs {
    const K* H;        // [NPAT]
    int j;             // 0, 1 or 2
    const K* chals;    // device row challenges r_0..r_{j-1}
    K beta1, beta2;    // beta_r[1], beta_r[2]
    K* partials;       // records [part_off + blockIdx.x]
    uint32_t part_off;
};

// Rounds 0..2: sum_P H[P] F_j(P, X) (one thread per canonical pattern).
__global__ void __launch_bounds__(FR) ccs_mom_round_kernel(const MomArgs a) {
    K c[REC];
#pragma unroll
    for (int d = 0; d < REC; d++) c[d] = gl::kzero();
    const int p = blockIdx.x * FR + threadIdx.x;
    if (p < NPAT) {
        const K h = a.H[p];
        if (!gl::kiszero(h)) {
            int tr[8];
            int P = p + NPAT + 1;
#pragma unroll
            for (int i = 0; i < 8; i++) { tr[i] = P % 3 - 1; P /= 3; }
            K F[4] = {gl::kzero(), gl::kzero(), gl::kzero(), gl::kzero()};
            if (a.j == 0) {
                // digits of pair s: lo = tr[2s], hi = tr[2s + 1]; weight chi_{beta1, beta2}(s)
                for (int s = 0; s < 4; s++) {
                    const int lo = tr[2 * s], b = tr[2 * s + 1] - lo;
                    const int n1 = b * (3 * lo * lo - 1), n2 = 3 * lo * b * b, n3 = b * b * b;
                    if (!(n1 | n2 | n3)) continue;
                    const K ws = gl::kmul((s & 1) ? a.beta1 : gl::ksub(gl::kone(), a.beta1),
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
                    n_coeffs(lo, hi, n);
                    if (j == 1) {
                        const K ws = s ? a.beta2 : gl::ksub(gl::kone(), a.beta2);
                        for (int d = 0; d < 4; d++) F[d] = gl::kadd(F[d], gl::kmul(ws, n[d]));
                    } else {
                        for (int d = 0; d < 4; d++) F[d] = n[d];
                    }
                }
            }
            for (int d = 0; d < 4; d++) c[d] = gl::kmul(h, F[d]);
        }
    }
    block_sum_rec(c, 4, a.partials + (uint64_t)(a.part_off + blockIdx.x) * REC);
}

struct FastRowArgs {
    // small tables: f variables at slots 1..n_fvar, eq_rin / eval at idx_eqrin / idx_eval
    const K* small_in;
    K* small_out;
    uint64_t small_len_in, small_len_out;
    int fold;
    K r;               // r_{j-1} (fold)
    int n_small;
    int idx_eqrin, idx_eval;
    FTerms f;
    int fdeg;          // degree of f (<= MAX_DEG - 1)
    const K* E;        // E_j [pairs]
    // NC
    int j;
    const K* chals;    // device r_0..r_{j-1}
    const int8_t* Z;   // [nq][m] (modes 3, 4)
    uint64_t m;
    const K* nc_in;    // mode 5: T_{j-1} [nq][nc_len_in]
    uint64_t nc_len_in;
    K* nc_out;         // modes 4, 5: T_j [nq][nc_len_out] (null in the last round)
    uint64_t nc_len_out;
    const K* wg;       // [nq]
    uint32_t nq, q_chunk, n_chunk;
    uint64_t pairs;
    K* partials;
    uint32_t part_off;
};

// Small tables of one row round: fold (rounds >= 1), f_t(X) and the eval
// term, for every pair t (one thread each).  Adds E_j(t) f_t(X) to S and
// eq_rin_t(X) eval_t(X) to V.
__global__ void __launch_bounds__(FR) ccs_fast_small_kernel(const FastRowArgs a) {
    K out[REC];
#pragma unroll
    for (int d = 0; d < REC; d++) out[d] = gl::kzero();
    const uint64_t t = blockIdx.x * (uint64_t)FR + threadIdx.x;
    if (t < a.pairs) {
        K lo_s[2 + MAX_FVAR + 2], hi_s[2 + MAX_FVAR + 2];
        for (int s = 1; s < a.n_small; s++) {
            K lo, hi;
            if (a.fold) {
                const K* in = a.small_in + (uint64_t)s * a.small_len_in + 4 * t;
                lo = gl::klerp(ld_k(in), ld_k(in + 1), a.r);
                hi = gl::klerp(ld_k(in + 2), ld_k(in + 3), a.r);
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
        K S[MAX_DEG];
#pragma unroll
        for (int d = 0; d < MAX_DEG; d++) S[d] = gl::kzero();
        for (int tt = 0; tt < a.f.n_terms; tt++) {
            K tp[MAX_DEG];
#pragma unroll
            for (int d = 0; d < MAX_DEG; d++) tp[d] = gl::kzero();
            tp[0] = a.f.coeff[tt];
            for (int vv = 0; vv < a.f.n_vars[tt]; vv++) {
                const int pos = a.f.var_pos[tt][vv];
                const K av = lo_s[1 + pos], bv = gl::ksub(hi_s[1 + pos], av);
                for (int e = 0; e < a.f.var_exp[tt][vv]; e++) {
                    K prev = gl::kzero();
#pragma unroll
                    for (int d = 0; d < MAX_DEG; d++) {
                        if (d <= a.fdeg) {
                            const K old = tp[d];
                            tp[d] = gl::kadd(gl::kmul(av, old), gl::kmul(bv, prev));
                            prev = old;
                        }
                    }
                }
            }
#pragma unroll
            for (int d = 0; d < MAX_DEG; d++) S[d] = gl::kadd(S[d], tp[d]);
        }
        const K e = a.E[t];
#pragma unroll
        for (int d = 0; d < MAX_DEG; d++)
            if (d <= a.fdeg) out[d] = gl::kmul(e, S[d]);
        if (a.idx_eval >= 0) {
            const K r0 = lo_s[a.idx_eqrin], r1 = gl::ksub(hi_s[a.idx_eqrin], r0);
            const K v0 = lo_s[a.idx_eval], v1 = gl::ksub(hi_s[a.idx_eval], v0);
            out[MAX_DEG] = gl::kmul(r0, v0);
            out[MAX_DEG + 1] = gl::kadd(gl::kmul(r0, v1), gl::kmul(r1, v0));
            out[MAX_DEG + 2] = gl::kmul(r1, v1);
        }
    }
    block_sum_rec(out, REC, a.partials + (uint64_t)(a.part_off + blockIdx.x) * REC);
}

// NC term of row rounds >= 3: MODE 3 / 4 stream 16- / 32-row digit blocks,
// MODE 5 folds the K table.  Thread = (pair t, q chunk c), t fastest; adds
// E_j(t) sum_{q in chunk} wg_q N(y_{q,t}(X)) to S.
template <int MODE>
__global__ void __launch_bounds__(FR, 2) ccs_fast_nc_kernel(const FastRowArgs a) {
    constexpr int NLUT = MODE == 3 ? 2 : (MODE == 4 ? 4 : 0);
    __shared__ K s_lut[NLUT ? NLUT * 81 : 1];
    __shared__ K s_w[16];
    extern __shared__ K s_wg[];  // [nq]
    const uint64_t gid = blockIdx.x * (uint64_t)FR + threadIdx.x;
    const bool live = gid < a.pairs * a.n_chunk;
    const uint64_t t = live ? gid % a.pairs : 0;
    const uint32_t c = live ? (uint32_t)(gid / a.pairs) : 0;
    if constexpr (NLUT > 0) {
        if (threadIdx.x < (1 << a.j)) s_w[threadIdx.x] = chi_of(a.chals, a.j, threadIdx.x);
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

    K out[4];
#pragma unroll
    for (int d = 0; d < 4; d++) out[d] = gl::kzero();
    if (live) {
        gl::KAcc acc[4];
#pragma unroll
        for (int d = 0; d < 4; d++) gl::kacc_zero(acc[d]);
        const uint32_t q0 = c * a.q_chunk, q1 = min(a.nq, q0 + a.q_chunk);
        for (uint32_t q = q0; q < q1; q++) {
            K lo, hi;
            if constexpr (MODE == 3) {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.Z + (uint64_t)q * a.m + 16 * t));
                if ((v.x | v.y | v.z | v.w) == 0) continue;
                lo = gl::kadd(s_lut[p4_index(v.x)], s_lut[81 + p4_index(v.y)]);
                hi = gl::kadd(s_lut[p4_index(v.z)], s_lut[81 + p4_index(v.w)]);
            } else if constexpr (MODE == 4) {
                const uint4* zp = reinterpret_cast<const uint4*>(a.Z + (uint64_t)q * a.m + 32 * t);
                const uint4 v = __ldg(zp), u = __ldg(zp + 1);
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
                const K* in = a.nc_in + (uint64_t)q * a.nc_len_in + 4 * t;
                const K x0 = ld_k(in), x1 = ld_k(in + 1), x2 = ld_k(in + 2), x3 = ld_k(in + 3);
                lo = gl::klerp(x0, x1, a.r);
                hi = gl::klerp(x2, x3, a.r);
                if (a.nc_out) {
                    K* o = a.nc_out + (uint64_t)q * a.nc_len_out + 2 * t;
                    st_k(o, lo);
                    st_k(o + 1, hi);
                }
                if (gl::kiszero(lo) && gl::kiszero(hi)) continue;
            }
            K n[4];
            n_coeffs(lo, hi, n);
            const K w = s_wg[q];
            const uint64_t w7 = gl::mul7(w.im);
#pragma unroll
            for (int d = 0; d < 4; d++) gl::kacc_mad(acc[d], w, w7, n[d]);
        }
        const K e = a.E[t];
#pragma unroll
        for (int d = 0; d < 4; d++) out[d] = gl::kmul(e, gl::kacc_reduce(acc[d]));
    }
    block_sum_rec(out, 4, a.partials + (uint64_t)(a.part_off + blockIdx.x) * REC);
}

struct FastReduceArgs {
    const K* partials;
    uint32_t nrec;
    int ncoef;          // deg_max + 1 coefficients written
    int j;
    const K* chals;     // device r_0..r_{j-1}
    K beta[32];         // beta_r
    K gamma_to_k;
    K* coeffs_out;
};

// p_j(X) = C_j eq(beta_j, X) S(X) + gamma^k V(X), coefficients low -> high.
__global__ void __launch_bounds__(256) ccs_fast_reduce_kernel(const FastReduceArgs a) {
    __shared__ K s_sum[REC];
    __shared__ K s_red[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d < REC; d++) {
        K v = gl::kzero();
        for (uint32_t b = threadIdx.x; b < a.nrec; b += blockDim.x) v = gl::kadd(v, a.partials[(uint64_t)b * REC + d]);
        for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_k(v, o));
        if (lane == 0) s_red[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            K s = gl::kzero();
            for (int w = 0; w < 8; w++) s = gl::kadd(s, s_red[w]);
            s_sum[d] = s;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        K Cj = gl::kone();
        for (int i = 0; i < a.j; i++) Cj = gl::kmul(Cj, eq_lin(a.beta[i], a.chals[i]));
        const K bj = a.beta[a.j];
        const K e0 = gl::kmul(Cj, gl::ksub(gl::kone(), bj));            // eq(beta_j, X) C_j = e0 + e1 X
        const K e1 = gl::kmul(Cj, gl::ksub(gl::kdbl(bj), gl::kone()));
        for (int d = 0; d < a.ncoef; d++) {
            K v = gl::kzero();
            if (d < MAX_DEG) v = gl::kmul(e0, s_sum[d]);
            if (d >= 1 && d - 1 < MAX_DEG) v = gl::kadd(v, gl::kmul(e1, s_sum[d - 1]));
            if (d < 3) v = gl::kadd(v, gl::kmul(a.gamma_to_k, s_sum[MAX_DEG + d]));
            a.coeffs_out[d] = v;
        }
    }
}
