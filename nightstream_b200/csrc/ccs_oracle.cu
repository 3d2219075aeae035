// ccs_oracle.cu -- Pi_CCS sum-check oracle (RoundOracle) on sm_100a.
//
// Reference: OptimizedOracle / RowStreamState
// (crates/neo-reductions/src/engines/optimized_engine/oracle.rs:82-503,
// 1047-1178, 1597-2104).  Round polynomial of the row phase, for pairs
// (2t, 2t+1) of every table (LSB-first binding):
//   p(X) = sum_t eq_br(X) * ( f(M z1)(X) + sum_{i,rho} wg[i,rho] N(y_{i,rho}(X)) )
//          + gamma^k * eq_rin(X) * eval(X),         N(y) = y^3 - y  (b = 2)
// computed as coefficients (low -> high) and evaluated at the requested xs.
//
// Design:
//  * Witness digit planes Z_i[rho][row] stay int8 in HBM.  For the first J
//    rounds the folded value of a table entry after j bound variables is
//    sum_b chi(r_0..r_{j-1})[b] * Z[rho][2^j t + b]: it is recomputed from the
//    digits each round (adds only) instead of materialising 16-byte K tables.
//  * Round J writes the K table T_J; later rounds read T_{j-1}, fold with
//    r_{j-1}, write T_j (ping-pong) and evaluate, all in one pass.
//  * The eq / f-variable / eval tables are folded the same way inside the
//    round kernel.  Block partial coefficients are reduced by a second kernel
//    in a fixed order, so results are deterministic (exact F_q arithmetic
//    makes them order-independent anyway).
#include "internal.cuh"
#include "tune.h"
#include <algorithm>
#include <cstdlib>
#include <memory>

using gl::K;

namespace {

constexpr int MAX_DEG = 8;    // deg_max + 1 <= 9 coefficients
constexpr int MAX_TERMS = 8;
constexpr int MAX_FVAR = 8;
constexpr int RT = 256;       // threads per round block
constexpr int JMAX = 4;       // rounds streamed from int8 digits (0..JMAX)

struct FTerms {
    int n_terms;
    int n_vars[MAX_TERMS];
    int var_pos[MAX_TERMS][4];
    int var_exp[MAX_TERMS][4];
    K coeff[MAX_TERMS];
};

struct RoundArgs {
    // small tables [n_small][len]
    const K* small_in;
    K* small_out;
    uint64_t small_len_in;
    uint64_t small_len_out;
    int fold;          // small_in must be folded by r first
    K r;
    int n_small;
    int n_fvar;
    int idx_eqrin;     // -1 when absent
    int idx_eval;      // -1 when absent
    K gamma_to_k;
    FTerms f;
    int deg_max;
    // NC
    const int8_t* Z;   // [nq][m]
    uint64_t m;
    const K* eqw;      // [2^j] chi of the bound prefix (streaming mode)
    const K* nc_in;    // K-mode input [nq][nc_len_in]
    uint64_t nc_len_in;
    K* nc_out;         // written table [nq][nc_len_out] or null
    uint64_t nc_len_out;
    const K* wg;       // [nq]
    int nq;
    int q_per_block;
    uint64_t pairs;
    K* partials;       // [gridDim.x * gridDim.y][deg_max+1]
};

__device__ __forceinline__ K shfl_xor_k(K a, int o) {
    K b;
    b.re = __shfl_xor_sync(0xffffffffu, a.re, o);
    b.im = __shfl_xor_sync(0xffffffffu, a.im, o);
    return b;
}

__device__ __forceinline__ K ld_k(const K* p) {
    ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
    return gl::kmk(v.x, v.y);
}
__device__ __forceinline__ void st_k(K* p, K a) {
    *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(a.re, a.im);
}

// N(a + bX) coefficients accumulated with weight wg into inner[0..3]
__device__ __forceinline__ void nc_accum_k(K wg, K a, K hi, K inner[4]) {
    K bb = gl::ksub(hi, a);
    K a2 = gl::ksqr(a);
    K a3 = gl::kmul(a2, a);
    K b2 = gl::ksqr(bb);
    K b3 = gl::kmul(b2, bb);
    K a2b = gl::kmul(a2, bb);
    K ab2 = gl::kmul(a, b2);
    K t0 = gl::ksub(a3, a);
    K t1 = gl::ksub(gl::kadd(gl::kdbl(a2b), a2b), bb);
    K t2 = gl::kadd(gl::kdbl(ab2), ab2);
    inner[0] = gl::kadd(inner[0], gl::kmul(wg, t0));
    inner[1] = gl::kadd(inner[1], gl::kmul(wg, t1));
    inner[2] = gl::kadd(inner[2], gl::kmul(wg, t2));
    inner[3] = gl::kadd(inner[3], gl::kmul(wg, b3));
}

// small-integer case (round 0): a = lo, hi are int8 digits, so every
// coefficient of N(a + bX) is a small integer (|.| < 2^25).
__device__ __forceinline__ void nc_accum_small(K wg, int a, int hi, K inner[4]) {
    int bb = hi - a;
    int t0 = a * a * a - a;             // 0 for a in {-1,0,1}
    int t1 = bb * (3 * a * a - 1);
    int t2 = 3 * a * bb * bb;
    int t3 = bb * bb * bb;
    if (t0) inner[0] = gl::kadd(inner[0], gl::kscale_small(wg, t0));
    if (t1) inner[1] = gl::kadd(inner[1], gl::kscale_small(wg, t1));
    if (t2) inner[2] = gl::kadd(inner[2], gl::kscale_small(wg, t2));
    if (t3) inner[3] = gl::kadd(inner[3], gl::kscale_small(wg, t3));
}

template <int NB>  // bytes per row pair = 2^(j+1)
__device__ __forceinline__ void load_digits(const int8_t* p, int8_t* d) {
    if constexpr (NB == 2) {
        char2 v = *reinterpret_cast<const char2*>(p);
        d[0] = v.x; d[1] = v.y;
    } else if constexpr (NB == 4) {
        char4 v = *reinterpret_cast<const char4*>(p);
        d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    } else if constexpr (NB == 8) {
        int2 v = __ldg(reinterpret_cast<const int2*>(p));
        memcpy(d, &v, 8);
    } else {
#pragma unroll
        for (int o = 0; o < NB; o += 16) {
            int4 v = __ldg(reinterpret_cast<const int4*>(p + o));
            memcpy(d + o, &v, 16);
        }
    }
}

// MODE 0..JMAX: digit streaming at round j = MODE; MODE = JMAX + 1: K tables.
template <int MODE>
__global__ void __launch_bounds__(RT) ccs_round_kernel(const RoundArgs a) {
    const uint64_t t = blockIdx.x * (uint64_t)RT + threadIdx.x;
    const bool live = t < a.pairs;
    const int dm = a.deg_max;
    K coeffs[MAX_DEG + 1];
#pragma unroll
    for (int d = 0; d <= MAX_DEG; d++) coeffs[d] = gl::kzero();

    __shared__ K s_wg[1024];
    __shared__ K s_eqw[1 << JMAX];
    const int q0 = blockIdx.y * a.q_per_block;
    const int q1 = min(a.nq, q0 + a.q_per_block);
    for (int q = q0 + threadIdx.x; q < q1; q += RT) s_wg[q - q0] = a.wg[q];
    if constexpr (MODE <= JMAX) {
        for (int b = threadIdx.x; b < (1 << MODE); b += RT) s_eqw[b] = a.eqw[b];
    }
    __syncthreads();

    if (live) {
        K inner[MAX_DEG + 1];
#pragma unroll
        for (int d = 0; d <= MAX_DEG; d++) inner[d] = gl::kzero();
        // ---- small tables: eq_beta_r, f vars, eq_rin, eval (only y-block 0) ----
        K e0 = gl::kzero(), e1 = gl::kzero();
        if (blockIdx.y == 0) {
            K lo_s[2 + MAX_FVAR + 2], hi_s[2 + MAX_FVAR + 2];
            for (int s = 0; s < a.n_small; s++) {
                K lo, hi;
                if (a.fold) {
                    const K* in = a.small_in + (uint64_t)s * a.small_len_in + 4 * t;
                    K x0 = ld_k(in), x1 = ld_k(in + 1), x2 = ld_k(in + 2), x3 = ld_k(in + 3);
                    lo = gl::klerp(x0, x1, a.r);
                    hi = gl::klerp(x2, x3, a.r);
                    if (a.small_out) {
                        K* out = a.small_out + (uint64_t)s * a.small_len_out + 2 * t;
                        st_k(out, lo);
                        st_k(out + 1, hi);
                    }
                } else {
                    const K* in = a.small_in + (uint64_t)s * a.small_len_in + 2 * t;
                    lo = ld_k(in);
                    hi = ld_k(in + 1);
                }
                lo_s[s] = lo;
                hi_s[s] = hi;
            }
            e0 = lo_s[0];
            e1 = gl::ksub(hi_s[0], e0);
            // f(X) = sum_terms coeff * prod (a_v + b_v X)^exp, truncated to deg_max+1
            for (int tt = 0; tt < a.f.n_terms; tt++) {
                K tp[MAX_DEG + 1];
#pragma unroll
                for (int d = 0; d <= MAX_DEG; d++) tp[d] = gl::kzero();
                tp[0] = a.f.coeff[tt];
                for (int vv = 0; vv < a.f.n_vars[tt]; vv++) {
                    int pos = a.f.var_pos[tt][vv];
                    K av = lo_s[1 + pos];
                    K bv = gl::ksub(hi_s[1 + pos], av);
                    for (int e = 0; e < a.f.var_exp[tt][vv]; e++) {
                        K prev = gl::kzero();
#pragma unroll
                        for (int d = 0; d <= MAX_DEG; d++) {
                            if (d <= dm) {
                                K old = tp[d];
                                tp[d] = gl::kadd(gl::kmul(av, old), gl::kmul(bv, prev));
                                prev = old;
                            }
                        }
                    }
                }
#pragma unroll
                for (int d = 0; d <= MAX_DEG; d++) inner[d] = gl::kadd(inner[d], tp[d]);
            }
            if (a.idx_eval >= 0) {
                K r0 = lo_s[a.idx_eqrin], r1 = gl::ksub(hi_s[a.idx_eqrin], r0);
                K v0 = lo_s[a.idx_eval], v1 = gl::ksub(hi_s[a.idx_eval], v0);
                K g = a.gamma_to_k;
                coeffs[0] = gl::kadd(coeffs[0], gl::kmul(g, gl::kmul(r0, v0)));
                coeffs[1] = gl::kadd(coeffs[1], gl::kmul(g, gl::kadd(gl::kmul(r0, v1), gl::kmul(r1, v0))));
                coeffs[2] = gl::kadd(coeffs[2], gl::kmul(g, gl::kmul(r1, v1)));
            }
        } else {
            // NC-only blocks still need eq_beta_r at this pair
            K lo, hi;
            if (a.fold) {
                const K* in = a.small_in + 4 * t;
                lo = gl::klerp(ld_k(in), ld_k(in + 1), a.r);
                hi = gl::klerp(ld_k(in + 2), ld_k(in + 3), a.r);
            } else {
                lo = ld_k(a.small_in + 2 * t);
                hi = ld_k(a.small_in + 2 * t + 1);
            }
            e0 = lo;
            e1 = gl::ksub(hi, lo);
        }

        // ---- NC block ----
        K nc[4] = {gl::kzero(), gl::kzero(), gl::kzero(), gl::kzero()};
        if constexpr (MODE == 0) {
            for (int q = q0; q < q1; q++) {
                int8_t d[2];
                load_digits<2>(a.Z + (uint64_t)q * a.m + 2 * t, d);
                if (a.nc_out) {
                    K* out = a.nc_out + (uint64_t)q * a.nc_len_out + 2 * t;
                    st_k(out, gl::kfq(gl::from_i64(d[0])));
                    st_k(out + 1, gl::kfq(gl::from_i64(d[1])));
                }
                nc_accum_small(s_wg[q - q0], d[0], d[1], nc);
            }
        } else if constexpr (MODE <= JMAX) {
            constexpr int HALF = 1 << MODE;
            constexpr int NB = 2 * HALF;
            for (int q = q0; q < q1; q++) {
                int8_t d[NB];
                load_digits<NB>(a.Z + (uint64_t)q * a.m + (uint64_t)NB * t, d);
                K lo = gl::kzero(), hi = gl::kzero();
#pragma unroll
                for (int b = 0; b < HALF; b++) {
                    if (d[b] == 1) lo = gl::kadd(lo, s_eqw[b]);
                    else if (d[b] == -1) lo = gl::ksub(lo, s_eqw[b]);
                    else if (d[b] != 0) lo = gl::kadd(lo, gl::kscale_small(s_eqw[b], d[b]));
                    if (d[HALF + b] == 1) hi = gl::kadd(hi, s_eqw[b]);
                    else if (d[HALF + b] == -1) hi = gl::ksub(hi, s_eqw[b]);
                    else if (d[HALF + b] != 0) hi = gl::kadd(hi, gl::kscale_small(s_eqw[b], d[HALF + b]));
                }
                if (a.nc_out) {
                    K* out = a.nc_out + (uint64_t)q * a.nc_len_out + 2 * t;
                    st_k(out, lo);
                    st_k(out + 1, hi);
                }
                nc_accum_k(s_wg[q - q0], lo, hi, nc);
            }
        } else {
            for (int q = q0; q < q1; q++) {
                const K* in = a.nc_in + (uint64_t)q * a.nc_len_in + 4 * t;
                K x0 = ld_k(in), x1 = ld_k(in + 1), x2 = ld_k(in + 2), x3 = ld_k(in + 3);
                K lo = gl::klerp(x0, x1, a.r);
                K hi = gl::klerp(x2, x3, a.r);
                if (a.nc_out) {
                    K* out = a.nc_out + (uint64_t)q * a.nc_len_out + 2 * t;
                    st_k(out, lo);
                    st_k(out + 1, hi);
                }
                nc_accum_k(s_wg[q - q0], lo, hi, nc);
            }
        }
#pragma unroll
        for (int d = 0; d < 4; d++) inner[d] = gl::kadd(inner[d], nc[d]);
        // coeffs += eq_br(X) * inner(X)
        coeffs[0] = gl::kadd(coeffs[0], gl::kmul(e0, inner[0]));
#pragma unroll
        for (int d = 1; d <= MAX_DEG; d++)
            if (d <= dm) coeffs[d] = gl::kadd(coeffs[d], gl::kadd(gl::kmul(e0, inner[d]), gl::kmul(e1, inner[d - 1])));
    }

    // ---- block reduction of coeffs[0..dm] ----
    __shared__ K s_red[RT / 32][MAX_DEG + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d <= MAX_DEG; d++) {
        if (d <= dm) {
            K v = coeffs[d];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_k(v, o));
            if (lane == 0) s_red[warp][d] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x <= dm) {
        K v = gl::kzero();
        for (int w = 0; w < RT / 32; w++) v = gl::kadd(v, s_red[w][threadIdx.x]);
        a.partials[((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * (dm + 1) + threadIdx.x] = v;
    }
}

struct EvalArgs {
    const K* partials;
    uint32_t nblocks;
    int ncoef;
    int nx;
    K xs[16];
    K* coeffs_out;
    K* ys_out;
};

__global__ void __launch_bounds__(256) reduce_eval_kernel(const EvalArgs a) {
    __shared__ K s_c[MAX_DEG + 1];
    __shared__ K s_red[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d < a.ncoef; d++) {
        K v = gl::kzero();
        for (uint32_t b = threadIdx.x; b < a.nblocks; b += blockDim.x) v = gl::kadd(v, a.partials[(uint64_t)b * a.ncoef + d]);
        for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_k(v, o));
        if (lane == 0) s_red[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            K s = gl::kzero();
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = gl::kadd(s, s_red[w]);
            s_c[d] = s;
            a.coeffs_out[d] = s;
        }
        __syncthreads();
    }
    if (threadIdx.x < a.nx) {
        K x = a.xs[threadIdx.x];
        K r = s_c[a.ncoef - 1];
        for (int d = a.ncoef - 2; d >= 0; d--) r = gl::kadd(gl::kmul(r, x), s_c[d]);
        a.ys_out[threadIdx.x] = r;
    }
}

// ---------------------------------------------------------------------------
// Table build kernels
// ---------------------------------------------------------------------------
// z1[c] = sum_rho b^rho Z_0[rho][c]  (oracle.rs:215-243)
__global__ void z1_kernel(const int8_t* __restrict__ Z, uint64_t m, uint32_t b, uint64_t* __restrict__ z1) {
    uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c >= m) return;
    uint64_t acc = 0, pw = 1;
    for (int rho = 0; rho < NEO_D; rho++) {
        int z = Z[(uint64_t)rho * m + c];
        if (z == 1) acc = gl::add(acc, pw);
        else if (z == -1) acc = gl::sub(acc, pw);
        else if (z) acc = gl::add(acc, gl::mul(pw, gl::from_i64(z)));
        pw = gl::mul(pw, b);
    }
    z1[c] = acc;
}

// out[r] = (M x)[r] for base-field x (CSR), or x[r] for the identity (oracle.rs:245-285)
__global__ void spmv_fq_kernel(const uint64_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
                               const uint64_t* __restrict__ val, int is_identity, uint32_t n, uint32_t m,
                               const uint64_t* __restrict__ x, uint64_t n_pad, K* __restrict__ out) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
    uint64_t acc = 0;
    if (r < n) {
        if (is_identity) {
            acc = r < m ? x[r] : 0;
        } else {
            for (uint64_t k = row_ptr[r]; k < row_ptr[r + 1]; k++) acc = gl::add(acc, gl::mul(val[k], x[col[k]]));
        }
    }
    out[r] = gl::kfq(acc);
}

// u[c] = sum_{i>=1} sum_rho gamma^i chi_alpha[rho] Z_i[rho][c]  (Eval table input, oracle.rs:320-390)
__global__ void eval_u_kernel(const int8_t* __restrict__ Z, uint64_t m, uint32_t k, const K* __restrict__ w,
                              K* __restrict__ u) {
    uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c >= m) return;
    K acc = gl::kzero();
    for (uint32_t i = 1; i < k; i++)
        for (int rho = 0; rho < NEO_D; rho++) {
            int z = Z[((uint64_t)i * NEO_D + rho) * m + c];
            if (z == 0) continue;
            K x = w[i * NEO_D + rho];
            acc = z == 1 ? gl::kadd(acc, x) : (z == -1 ? gl::ksub(acc, x) : gl::kadd(acc, gl::kscale_small(x, z)));
        }
    u[c] = acc;
}

// u[c] of eval_u_kernel for ternary digit rows: the rows of instances 1..k-1
// taken in pairs (q, q+1), whose 9 signed weight sums +-w[q] +- w[q+1] sit in
// shared memory (the weights are the same for every column).  Thread = column,
// blockIdx.y = a range of row pairs: one table entry per row pair added
// unreduced in 128 bits; the last block of a column block (ticket) adds the
// ranges' partials.
constexpr uint32_t EU_MAX_PAIRS = 324;  // k <= 13
constexpr uint32_t EU_SPLIT = 8;
__global__ void __launch_bounds__(256) eval_u_pair_kernel(const int8_t* __restrict__ Z, uint64_t m, uint32_t k,
                                                          const K* __restrict__ w, K* __restrict__ partials,
                                                          unsigned int* __restrict__ tickets, K* __restrict__ u) {
    __shared__ K tab[EU_MAX_PAIRS / EU_SPLIT + 1][9];
    const uint32_t np = (k - 1) * NEO_D / 2;
    const uint32_t per = (np + gridDim.y - 1) / gridDim.y;
    const uint32_t g0 = blockIdx.y * per, g1 = min(np, g0 + per);
    for (uint32_t i = threadIdx.x; i < (g1 > g0 ? g1 - g0 : 0) * 9; i += blockDim.x) {
        const uint32_t g = g0 + i / 9, e = i % 9, q = NEO_D + 2 * g;
        const K a = w[q], b = w[q + 1];
        const uint32_t d0 = e % 3, d1 = e / 3;
        K s2 = d0 == 0 ? gl::kneg(a) : (d0 == 2 ? a : gl::kzero());
        tab[i / 9][e] = d1 == 0 ? gl::ksub(s2, b) : (d1 == 2 ? gl::kadd(s2, b) : s2);
    }
    __syncthreads();
    const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c < m) {
        uint64_t lo0 = 0, hi0 = 0, lo1 = 0, hi1 = 0;
        for (uint32_t g = g0; g < g1; g++) {
            const uint64_t q = NEO_D + 2 * (uint64_t)g;
            const int d0 = Z[q * m + c], d1 = Z[(q + 1) * m + c];
            const K x = tab[g - g0][(uint32_t)(d0 + 1) + 3u * (uint32_t)(d1 + 1)];
            lo0 += x.re;
            hi0 += lo0 < x.re;
            lo1 += x.im;
            hi1 += lo1 < x.im;
        }
        K r;
        r.re = gl::add(gl::canon(lo0), hi0 * 0xFFFFFFFFull);
        r.im = gl::add(gl::canon(lo1), hi1 * 0xFFFFFFFFull);
        partials[(uint64_t)blockIdx.y * m + c] = r;
    }
    __threadfence();
    __syncthreads();
    __shared__ unsigned int s_last;
    if (threadIdx.x == 0) s_last = atomicInc(tickets + blockIdx.x, gridDim.y - 1) == gridDim.y - 1;
    __syncthreads();
    if (!s_last || c >= m) return;
    __threadfence();
    K a = gl::kzero();
    for (uint32_t sp = 0; sp < gridDim.y; sp++) {
        const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(partials + (uint64_t)sp * m + c));
        a = gl::kadd(a, gl::kmk(v.x, v.y));
    }
    u[c] = a;
}

// eval[r] = sum_j coef_j (M_j u)[r]
__global__ void eval_tbl_kernel(const uint64_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
                                const uint64_t* __restrict__ val, const uint64_t* __restrict__ nnz_off,
                                const uint8_t* __restrict__ is_id, uint32_t t, uint32_t n, uint32_t m,
                                const K* __restrict__ u, const K* __restrict__ coef, uint64_t n_pad,
                                K* __restrict__ out) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
    K acc = gl::kzero();
    if (r < n) {
        for (uint32_t j = 0; j < t; j++) {
            K mj = gl::kzero();
            if (is_id[j]) {
                if (r < m) mj = u[r];
            } else {
                const uint64_t* rp = row_ptr + (uint64_t)j * (n + 1);
                uint64_t base = nnz_off[j];
                for (uint64_t k = rp[r]; k < rp[r + 1]; k++)
                    mj = gl::kadd(mj, gl::kscale(u[col[base + k]], val[base + k]));
            }
            acc = gl::kadd(acc, gl::kmul(coef[j], mj));
        }
    }
    out[r] = acc;
}

// ---------------------------------------------------------------------------
// Ajtai phase (oracle.rs:1812-1951): one block.
// ---------------------------------------------------------------------------
struct AjtaiArgs {
    int k, t, ell_d, ell_n, j, nx, has_inputs;
    K xs[16];
    K alpha[8], beta_a[8], ajtai_chals[8];
    K beta_r[32], r_in[32], row_chals[32];
    K gamma;
    FTerms f;
    int fvar_j[MAX_FVAR];
    const K* y;      // [k][t][54]
    const K* ysc;    // [k][t]
    K* ys_out;       // [nx]
};

__device__ K eq_lin_d(K a, K b) {
    return gl::kadd(gl::kmul(gl::ksub(gl::kone(), a), gl::ksub(gl::kone(), b)), gl::kmul(a, b));
}

// warp-wide sum of K values (lane 0 holds the total)
__device__ __forceinline__ K warp_ksum(K v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        K o;
        o.re = __shfl_down_sync(0xffffffffu, (unsigned long long)v.re, off);
        o.im = __shfl_down_sync(0xffffffffu, (unsigned long long)v.im, off);
        v = gl::kadd(v, o);
    }
    return v;
}

// One Ajtai-phase round (oracle.rs:1659-1953): evaluations at xs of round j
// over the 54 (padded to 2^ell_d) Ajtai coordinates.  Field arithmetic is
// exact, so the work is reordered for parallelism without changing a bit:
//  * the prefix fold by bits 0..j-1 of each vector is the weighted sum with
//    the chi weights of those challenges (one thread per folded entry);
//  * an evaluation vector's round value is linear in x, A + (B - A) x with
//    A, B the tail-weighted sums of its lo / hi entries, so its gamma-weighted
//    combination is formed once per round, not once per x;
//  * x-independent products (gamma powers, prefix and row equalities, F') are
//    separate threads' chains, and tail sums are warp reductions.
__global__ void __launch_bounds__(512) ajtai_round_kernel(const AjtaiArgs a) {
    extern __shared__ K s_dyn[];          // s_y [nvec][54] folded, then s_nc [nx][k]
    __shared__ K s_wb[128], s_wa[128], s_w[128];
    __shared__ K s_A[160], s_B[160];
    __shared__ K s_gp[161];               // gamma^0..gamma^k
    __shared__ K s_gkp[160];              // (gamma^k)^0..(gamma^k)^(t-1), t < k (1 + t) <= 160
    __shared__ K s_fixed[8];              // ebp, eap, eq_br, eq_ri, fprime, SA, SB
    __shared__ K s_ncsum[16];
    const int nvec = a.k * (1 + a.t);     // vector q < k: NC (y[i][0]); then eval (i, jm)
    K* s_y = s_dyn;
    K* s_nc = s_dyn + nvec * NEO_D;
    const int j = a.j, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int ntail = a.ell_d - j - 1, tail_len = 1 << ntail;
    const int hs = 1 << (j + 1), stride = 1 << j;

    // ---- 1. x-independent chains and weights ----
    if (tid == 0) {
        K g = gl::kone();
        s_gp[0] = g;
        for (int i = 0; i < a.k; i++) { g = gl::kmul(g, a.gamma); s_gp[i + 1] = g; }
        K p = gl::kone();
        for (int jm = 0; jm < a.t; jm++) { s_gkp[jm] = p; p = gl::kmul(p, g); }
    } else if (tid == 1 || tid == 2) {
        K e = gl::kone();
        for (int i = 0; i < j; i++) e = gl::kmul(e, eq_lin_d(a.ajtai_chals[i], tid == 1 ? a.beta_a[i] : a.alpha[i]));
        s_fixed[tid - 1] = e;  // ebp, eap
    } else if (tid == 3 || tid == 4) {
        K e = gl::kone();
        if (tid == 3 || a.has_inputs)
            for (int i = 0; i < a.ell_n; i++) e = gl::kmul(e, eq_lin_d(a.row_chals[i], tid == 3 ? a.beta_r[i] : a.r_in[i]));
        s_fixed[tid - 1] = e;  // eq_br, eq_ri
    } else if (tid == 5) {
        // F' = f(m_vals), m_vals[j] = y_scalars[0][j] (z1 . v_j by linearity of recomposition)
        K fprime = gl::kzero();
        for (int tt = 0; tt < a.f.n_terms; tt++) {
            K p = a.f.coeff[tt];
            for (int vv = 0; vv < a.f.n_vars[tt]; vv++) {
                K mv = a.ysc[a.fvar_j[a.f.var_pos[tt][vv]]];
                for (int e = 0; e < a.f.var_exp[tt][vv]; e++) p = gl::kmul(p, mv);
            }
            fprime = gl::kadd(fprime, p);
        }
        s_fixed[4] = fprime;
    } else if (tid >= 32 && tid < 32 + (1 << j)) {
        // fold weight of offset b: prod over bits of (bit ? c : 1 - c)
        const int b = tid - 32;
        K w = gl::kone();
        for (int i = 0; i < j; i++) w = gl::kmul(w, ((b >> i) & 1) ? a.ajtai_chals[i] : gl::ksub(gl::kone(), a.ajtai_chals[i]));
        s_w[b] = w;
    } else if (tid >= 160 && tid < 160 + tail_len) {
        // tail weights chi(beta_a[j+1..]), chi(alpha[j+1..])
        const int tt = tid - 160;
        K wb = gl::kone(), wa = gl::kone();
        for (int i = 0; i < ntail; i++) {
            int bit = (tt >> i) & 1;
            K b = a.beta_a[j + 1 + i], al = a.alpha[j + 1 + i];
            wb = gl::kmul(wb, bit ? b : gl::ksub(gl::kone(), b));
            wa = gl::kmul(wa, bit ? al : gl::ksub(gl::kone(), al));
        }
        s_wb[tt] = wb;
        s_wa[tt] = wa;
    }
    __syncthreads();

    // ---- 2. prefix fold by bits 0..j-1: entry i of the folded vector at s_y[q][i 2^j] ----
    {
        const int L = (NEO_D + stride - 1) >> j;
        for (int w = tid; w < nvec * L; w += blockDim.x) {
            const int q = w / L, i = w % L;
            const K* src = q < a.k ? a.y + ((uint64_t)q * a.t + 0) * NEO_D : a.y + (uint64_t)(q - a.k) * NEO_D;
            const int base = i << j;
            K acc;
            if (j == 0) {
                acc = src[base];
            } else {
                acc = gl::kzero();
                for (int b = 0; b < stride && base + b < NEO_D; b++) acc = gl::kadd(acc, gl::kmul(s_w[b], src[base + b]));
            }
            s_y[q * NEO_D + base] = acc;
        }
    }
    __syncthreads();

    // ---- 3. tail sums: `seg` lanes per item (the tail length, at most 32),
    //         32 / seg items per warp, segment sums by width-limited shuffles ----
    const int n_nc = a.nx * a.k, n_items = n_nc + 2 * (nvec - a.k);
    const int seg = tail_len < 32 ? tail_len : 32, per_warp = 32 / seg;
    const int sub = lane % seg;
    for (int base = warp * per_warp; base < n_items; base += nwarps * per_warp) {
        const int item = base + lane / seg;
        K part = gl::kzero();
        if (item < n_nc) {
            const int xi = item / a.k, q = item % a.k;
            const K x = a.xs[xi];
            const K* v = s_y + q * NEO_D;
            for (int tt = sub; tt < tail_len; tt += seg) {
                const int idx = tt * hs;
                if (idx >= NEO_D) continue;
                const int i1 = idx + stride;
                K val = gl::klerp(v[idx], i1 < NEO_D ? v[i1] : gl::kzero(), x);
                val = gl::kmul(val, gl::ksub(gl::ksqr(val), gl::kone()));  // range product, b = 2
                part = gl::kadd(part, gl::kmul(s_wb[tt], val));
            }
        } else if (item < n_items) {
            const int e = item - n_nc, q = a.k + (e >> 1), hi_side = e & 1;
            const K* v = s_y + q * NEO_D;
            for (int tt = sub; tt < tail_len; tt += seg) {
                const int idx = tt * hs;
                if (idx >= NEO_D) continue;
                const int pos = idx + (hi_side ? stride : 0);
                if (pos < NEO_D) part = gl::kadd(part, gl::kmul(s_wa[tt], v[pos]));
            }
        }
        for (int off = seg >> 1; off > 0; off >>= 1) {
            K o;
            o.re = __shfl_down_sync(0xffffffffu, (unsigned long long)part.re, off, seg);
            o.im = __shfl_down_sync(0xffffffffu, (unsigned long long)part.im, off, seg);
            part = gl::kadd(part, o);
        }
        if (sub == 0 && item < n_items) {
            if (item < n_nc) {
                s_nc[(item / a.k) * a.k + item % a.k] = part;
            } else {
                const int e = item - n_nc;
                (e & 1 ? s_B : s_A)[a.k + (e >> 1)] = part;
            }
        }
    }
    __syncthreads();

    // ---- 4. gamma-weighted combinations ----
    if (warp == 0 || warp == 1) {
        // S = sum_{jm, i >= 1} gamma^i (gamma^k)^jm X[k + i t + jm], X = A (warp 0) or B (warp 1)
        const K* X = warp == 0 ? s_A : s_B;
        const int nterm = (a.k - 1) * a.t;
        K part = gl::kzero();
        for (int u = lane; u < nterm; u += 32) {
            const int i = 1 + u / a.t, jm = u % a.t;
            part = gl::kadd(part, gl::kmul(gl::kmul(s_gp[i], s_gkp[jm]), X[a.k + i * a.t + jm]));
        }
        part = warp_ksum(part);
        if (lane == 0) s_fixed[5 + warp] = part;
    } else {
        // nc_sum[x] = sum_i gamma^(i+1) nc[x][i], warps 2.. over the points
        for (int xi = warp - 2; xi < a.nx; xi += nwarps - 2) {
            K part = gl::kzero();
            for (int i = lane; i < a.k; i += 32) part = gl::kadd(part, gl::kmul(s_gp[i + 1], s_nc[xi * a.k + i]));
            part = warp_ksum(part);
            if (lane == 0) s_ncsum[xi] = part;
        }
    }
    __syncthreads();

    // ---- 5. per evaluation point ----
    if (tid < a.nx) {
        const int xi = tid;
        const K x = a.xs[xi];
        const K gk = s_gp[a.k];
        const K eq_beta = gl::kmul(s_fixed[2], gl::kmul(s_fixed[0], eq_lin_d(x, a.beta_a[j])));
        const K eq_ar = a.has_inputs ? gl::kmul(s_fixed[3], gl::kmul(s_fixed[1], eq_lin_d(x, a.alpha[j]))) : gl::kzero();
        K out = gl::kmul(eq_beta, gl::kadd(s_fixed[4], s_ncsum[xi]));
        if (a.k >= 2 && !gl::kiszero(eq_ar)) {
            const K inner = gl::klerp(s_fixed[5], s_fixed[6], x);
            out = gl::kadd(out, gl::kmul(eq_ar, gl::kmul(gk, inner)));
        }
        a.ys_out[xi] = out;
    }
}

#include "ccs_fast.cuh"

}  // namespace

// ---------------------------------------------------------------------------
// Oracle object
// ---------------------------------------------------------------------------
struct neo_gpu_ccs_oracle {
    neo_gpu_ctx* ctx = nullptr;
    uint32_t k = 0, b = 2, ell_d = 0, ell_n = 0, d_sc = 0, t = 0;
    uint64_t n_pad = 0, m = 0;
    DevCcs own_ccs;          // used when the oracle owns its CCS copy
    const DevCcs* ccs = nullptr;
    DevBuf<int8_t> own_Z;    // used when the oracle owns its witness copy
    const int8_t* Z = nullptr;
    FTerms f{};
    int n_fvar = 0;
    int fvar_j[MAX_FVAR] = {0};
    int deg_max = 4;
    int n_small = 0, idx_eqrin = -1, idx_eval = -1;
    DevBuf<K> small[2];
    int small_cur = 0;
    DevBuf<K> nc[2];
    int nc_cur = 0;
    int J = 0;
    DevBuf<K> wg, eqw, partials, coeffs, ys, scratch_k;
    DevBuf<K> d_chals;  // row challenges on the device (prefix χ tables of the streaming rounds)
    // ternary-digit path (ccs_fast.cuh): E tables, the 8-row pattern histogram
    bool fast = false;
    DevBuf<K> E_all;            // E_j = chi_{beta_{j+1..}} at offset 2^ell - 2^(ell - j), j < ell
    DevBuf<uint64_t> hist64;    // [8][NPAT] limb sums of the pattern histogram
    DevBuf<uint32_t> hist_part; // [hist blocks][8][NPAT]
    DevBuf<uint32_t> tern_flag;
    DevBuf<uint32_t> ticket;    // last-block ticket of the fused round kernel
    DevBuf<K> Cs;               // C_j = prod_{i<j} eq(beta_i, r_i) per row round
    HostBuf<K> h_chals;         // page-locked staging of the row challenges (async upload)
    uint32_t hist_gx = 0, hist_gy = 0, hist_qc = 0;
    bool hist_split = false;
    uint32_t compact_q = 8;     // q per thread below which the NC blocks use out-of-line K products
    uint64_t nc_threads = 148ull * 2 * 256;  // NC threads per round (one wave) when the pairs alone are fewer
    uint64_t late_pairs = 0;                 // rounds with fewer pairs than this use late_threads NC threads
    uint64_t late_threads = 256;
    uint32_t hist_items = 16384;              // target (q, 8-row block) items per histogram block
    K gamma{}, gamma_to_k{};
    std::vector<K> alpha, beta_a, beta_r, r_in, row_chals, ajtai_chals;
    bool has_inputs = false, has_eval = false;
    uint32_t round_idx = 0;
    bool coeffs_valid = false;
    std::vector<K> h_coeffs;
    // Ajtai-phase state
    bool have_pre = false;
    DevBuf<K> chi_r, vj, y_eval, y_sc;
    // build temporaries, kept across re-initialisations
    DevBuf<K> ws_bits, ws_w, ws_coef, ws_u, ws_upart;  // ws_upart: eval_u_pair_kernel partials
    DevBuf<unsigned int> ws_uticket;
    DevBuf<uint64_t> ws_z1, ws_nnzoff;
    DevBuf<uint8_t> ws_isid;
};

static std::vector<K> load_k(const uint64_t* p, size_t n) {
    std::vector<K> v(n);
    for (size_t i = 0; i < n; i++) v[i] = gl::kmk(gl::canon(p[2 * i]), gl::canon(p[2 * i + 1]));
    return v;
}

static K host_chi_mask(size_t mask, const std::vector<K>& pts) {
    K p = gl::kone();
    for (size_t i = 0; i < pts.size(); i++) p = gl::kmul(p, ((mask >> i) & 1) ? pts[i] : gl::ksub(gl::kone(), pts[i]));
    return p;
}

static int oracle_init(neo_gpu_ctx* ctx, neo_gpu_ccs_oracle* o, const int8_t* d_Z, uint32_t k, uint32_t b,
                       const K* alpha, const K* beta_a, const K* beta_r, K gamma, const K* r_inputs,
                       uint32_t ell_d, uint32_t ell_n, uint32_t d_sc);
static int fast_setup(neo_gpu_ccs_oracle* o);

static int neo_gpu_ccs_oracle_create_impl_abi(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, const int8_t* Z, uint32_t k,
                                         uint32_t b, const uint64_t* alpha, const uint64_t* beta_a,
                                         const uint64_t* beta_r, const uint64_t* gamma, const uint64_t* r_inputs,
                                         uint32_t ell_d, uint32_t ell_n, uint32_t d_sc, neo_gpu_ccs_oracle** out) {
    if (!ctx) return NEO_ERR_ARG;
    if (!out || !desc || !Z || !alpha || !beta_a || !beta_r || !gamma) return ctx->fail(NEO_ERR_ARG, "ccs_oracle: null argument");
    *out = nullptr;
    if (ell_d == 0 || ell_d > 8 || ell_n < 1 || ell_n > 30) return ctx->fail(NEO_ERR_ARG, "ccs_oracle: ell_d/ell_n out of range");
    cudaSetDevice(ctx->device);
    auto* o = new neo_gpu_ccs_oracle();
    std::unique_ptr<neo_gpu_ccs_oracle> guard(o);
    int rc = dev_ccs_upload(ctx, desc, o->own_ccs);
    if (rc) return rc;
    o->ccs = &o->own_ccs;
    if (k == 0 || k > 18) return ctx->fail(NEO_ERR_ARG, "ccs_oracle: k must be in 1..18");
    NEO_CK(ctx, o->own_Z.alloc((size_t)k * NEO_D * desc->m));
    NEO_CK(ctx, cudaMemcpyAsync(o->own_Z.p, Z, o->own_Z.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    std::vector<K> al = load_k(alpha, ell_d), ba = load_k(beta_a, ell_d), br = load_k(beta_r, ell_n);
    std::vector<K> ri;
    if (r_inputs) ri = load_k(r_inputs, ell_n);
    rc = oracle_init(ctx, o, o->own_Z.p, k, b, al.data(), ba.data(), br.data(), load_k(gamma, 1)[0],
                     r_inputs ? ri.data() : nullptr, ell_d, ell_n, d_sc);
    if (rc) return rc;
    *out = guard.release();
    return NEO_OK;
}
extern "C" int neo_gpu_ccs_oracle_create(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, const int8_t* Z, uint32_t k,
                                         uint32_t b, const uint64_t* alpha, const uint64_t* beta_a,
                                         const uint64_t* beta_r, const uint64_t* gamma, const uint64_t* r_inputs,
                                         uint32_t ell_d, uint32_t ell_n, uint32_t d_sc, neo_gpu_ccs_oracle** out) { NEO_ABI_GUARD(neo_gpu_ccs_oracle_create_impl_abi(ctx, desc, Z, k, b, alpha, beta_a, beta_r, gamma, r_inputs, ell_d, ell_n, d_sc, out)) }

// Builds the oracle in *inout; an existing oracle is re-initialised in place so
// its device workspaces are reused across fold steps.
int ccs_oracle_create_dev(neo_gpu_ctx* ctx, const DevCcs* ccs, const int8_t* d_Z, uint32_t k, uint32_t b,
                          const K* alpha, const K* beta_a, const K* beta_r, K gamma, const K* r_inputs,
                          uint32_t ell_d, uint32_t ell_n, uint32_t d_sc, neo_gpu_ccs_oracle** inout) {
    std::unique_ptr<neo_gpu_ccs_oracle> guard;
    neo_gpu_ccs_oracle* o = *inout;
    if (!o) {
        o = new neo_gpu_ccs_oracle();
        guard.reset(o);
    }
    o->ccs = ccs;
    int rc = oracle_init(ctx, o, d_Z, k, b, alpha, beta_a, beta_r, gamma, r_inputs, ell_d, ell_n, d_sc);
    if (rc) return rc;
    if (guard) *inout = guard.release();
    return NEO_OK;
}

static int oracle_init(neo_gpu_ctx* ctx, neo_gpu_ccs_oracle* o, const int8_t* d_Z, uint32_t k, uint32_t b,
                       const K* alpha, const K* beta_a, const K* beta_r, K gamma, const K* r_inputs,
                       uint32_t ell_d, uint32_t ell_n, uint32_t d_sc) {
    const DevCcs& cc = *o->ccs;
    if (b != 2) return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_oracle: only b = 2 is implemented");
    if (k == 0 || k > 18) return ctx->fail(NEO_ERR_ARG, "ccs_oracle: k must be in 1..18");
    if (ell_d == 0 || ell_d > 8 || (1u << ell_d) < NEO_D) return ctx->fail(NEO_ERR_ARG, "ccs_oracle: ell_d");
    if (ell_n < 1 || ell_n > 30) return ctx->fail(NEO_ERR_ARG, "ccs_oracle: ell_n");
    if (cc.n != cc.m || cc.n != (1u << ell_n))
        return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_oracle: requires n == m == 2^ell_n");
    if (!cc.is_identity[0]) return ctx->fail(NEO_ERR_ARG, "ccs_oracle: CCS must be identity-first");
    o->ctx = ctx;
    o->Z = d_Z;
    o->k = k; o->b = b; o->ell_d = ell_d; o->ell_n = ell_n; o->d_sc = d_sc;
    // (re)initialisation: protocol state starts over, device buffers are reused
    o->f = FTerms{};
    o->n_fvar = 0;
    o->n_small = 0; o->idx_eqrin = -1; o->idx_eval = -1;
    o->small_cur = 0; o->nc_cur = 0;
    o->row_chals.clear(); o->ajtai_chals.clear(); o->r_in.clear();
    o->round_idx = 0; o->coeffs_valid = false; o->have_pre = false;
    int rc = 0;
    o->t = cc.t;
    o->m = cc.m;
    o->n_pad = 1ULL << ell_n;
    o->alpha.assign(alpha, alpha + ell_d);
    o->beta_a.assign(beta_a, beta_a + ell_d);
    o->beta_r.assign(beta_r, beta_r + ell_n);
    o->gamma = gamma;
    o->has_inputs = r_inputs != nullptr;
    if (o->has_inputs) o->r_in.assign(r_inputs, r_inputs + ell_n);
    o->has_eval = o->has_inputs && k >= 2;
    // every digit in {-1, 0, 1}?  Ternary digits (every witness the fold step
    // builds: balanced base-2 decomposition and split_b) take the
    // pattern-histogram row rounds and the pair-table kernels; any other digit
    // keeps the streaming kernels
    uint32_t h_bad = 1;
    if (ell_n >= 3) {
        NEO_CK(ctx, o->tern_flag.ensure(1));
        NEO_CK(ctx, cudaMemsetAsync(o->tern_flag.p, 0, 4, ctx->stream));
        const uint64_t nbytes = (uint64_t)k * NEO_D * cc.m;
        ternary_check_kernel<<<148 * 4, 256, 0, ctx->stream>>>(reinterpret_cast<const uint4*>(o->Z), nbytes / 16,
                                                              reinterpret_cast<const uint8_t*>(o->Z) + nbytes / 16 * 16,
                                                              (uint32_t)(nbytes % 16), o->tern_flag.p);
        NEO_LAUNCHED(ctx);
        NEO_CK(ctx, ctx_d2h(ctx, &h_bad, o->tern_flag.p, 4));
    }
    NEO_CK(ctx, ctx_sync(ctx));
    o->fast = h_bad == 0;
    struct { uint32_t n, m, n_terms; const uint32_t* f_exps; const uint64_t* f_coeff; } dd{
        cc.n, cc.m, cc.n_terms, cc.f_exps.data(), cc.f_coeff.data()};
    const auto* desc = &dd;

    // compile f (oracle.rs:136-186)
    const uint32_t t = o->t;
    std::vector<int> pos_by_j(t, -1);
    for (uint32_t j = 0; j < t; j++) {
        bool used = false;
        for (uint32_t tt = 0; tt < desc->n_terms; tt++) used |= desc->f_exps[tt * t + j] != 0;
        if (used) {
            if (o->n_fvar >= MAX_FVAR) return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_oracle: too many f variables");
            pos_by_j[j] = o->n_fvar;
            o->fvar_j[o->n_fvar++] = (int)j;
        }
    }
    if (desc->n_terms > MAX_TERMS) return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_oracle: too many f terms");
    int fmax = 0;
    o->f.n_terms = (int)desc->n_terms;
    for (uint32_t tt = 0; tt < desc->n_terms; tt++) {
        int dg = 0, nv = 0;
        o->f.coeff[tt] = gl::kfq(gl::canon(desc->f_coeff[tt]));
        for (uint32_t j = 0; j < t; j++) {
            uint32_t e = desc->f_exps[tt * t + j];
            if (!e) continue;
            if (nv >= 4) return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_oracle: term with more than 4 variables");
            o->f.var_pos[tt][nv] = pos_by_j[j];
            o->f.var_exp[tt][nv] = (int)e;
            nv++;
            dg += (int)e;
        }
        o->f.n_vars[tt] = nv;
        fmax = std::max(fmax, dg);
    }
    o->deg_max = std::max(4, fmax + 1);
    if (o->deg_max > MAX_DEG) return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_oracle: f degree too large");

    const uint64_t n_pad = o->n_pad, m = o->m;
    const uint32_t nq = k * NEO_D;

    // small tables: [0] eq_beta_r, [1..n_fvar] f vars, then eq_rin, eval
    o->n_small = 1 + o->n_fvar;
    if (o->has_eval) {
        o->idx_eqrin = o->n_small++;
        o->idx_eval = o->n_small++;
    }
    NEO_CK(ctx, o->small[0].ensure((size_t)o->n_small * n_pad));
    NEO_CK(ctx, o->small[1].ensure((size_t)o->n_small * n_pad / 2 + 1));
    K* S = o->small[0].p;
    DevBuf<K>& dbits = o->ws_bits;
    NEO_CK(ctx, dbits.ensure(2 * ell_n));
    NEO_CK(ctx, cudaMemcpyAsync(dbits.p, o->beta_r.data(), ell_n * 16, cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = launch_chi_table(ctx, dbits.p, ell_n, S))) return rc;
    DevBuf<uint64_t>& z1 = o->ws_z1;
    NEO_CK(ctx, z1.ensure(m));
    z1_kernel<<<ceil_div(m, 256), 256, 0, ctx->stream>>>(o->Z, m, b, z1.p);
    NEO_LAUNCHED(ctx);
    for (int v = 0; v < o->n_fvar; v++) {
        int j = o->fvar_j[v];
        spmv_fq_kernel<<<ceil_div(n_pad, 256), 256, 0, ctx->stream>>>(
            o->ccs->csr_ptr.p + (size_t)j * (desc->n + 1), o->ccs->csr_col.p + o->ccs->nnz_off[j],
            o->ccs->csr_val.p + o->ccs->nnz_off[j], o->ccs->is_identity[j], desc->n, desc->m, z1.p, n_pad,
            S + (size_t)(1 + v) * n_pad);
        NEO_LAUNCHED(ctx);
    }
    // gamma^k, wg
    o->gamma_to_k = gl::kone();
    for (uint32_t i = 0; i < k; i++) o->gamma_to_k = gl::kmul(o->gamma_to_k, o->gamma);
    std::vector<K> wg(nq);
    {
        K g = o->gamma;
        for (uint32_t i = 0; i < k; i++) {
            for (int rho = 0; rho < NEO_D; rho++) wg[i * NEO_D + rho] = gl::kmul(host_chi_mask(rho, o->beta_a), g);
            g = gl::kmul(g, o->gamma);
        }
    }
    NEO_CK(ctx, o->wg.ensure(nq));
    NEO_CK(ctx, cudaMemcpyAsync(o->wg.p, wg.data(), nq * 16, cudaMemcpyHostToDevice, ctx->stream));
    if (o->has_eval) {
        NEO_CK(ctx, cudaMemcpyAsync(dbits.p + ell_n, o->r_in.data(), ell_n * 16, cudaMemcpyHostToDevice, ctx->stream));
        if ((rc = launch_chi_table(ctx, dbits.p + ell_n, ell_n, S + (size_t)o->idx_eqrin * n_pad))) return rc;
        // w[i*54+rho] = gamma^i chi_alpha[rho]
        std::vector<K> w((size_t)nq), coef(t);
        K gi = gl::kone();
        for (uint32_t i = 0; i < k; i++) {
            for (int rho = 0; rho < NEO_D; rho++) w[i * NEO_D + rho] = i ? gl::kmul(gi, host_chi_mask(rho, o->alpha)) : gl::kzero();
            gi = gl::kmul(gi, o->gamma);
        }
        K gkj = gl::kone();
        for (uint32_t j = 0; j < t; j++) { coef[j] = gkj; gkj = gl::kmul(gkj, o->gamma_to_k); }
        DevBuf<K>& dw = o->ws_w;
        DevBuf<K>& dcoef = o->ws_coef;
        DevBuf<K>& du = o->ws_u;
        NEO_CK(ctx, dw.ensure(nq));
        NEO_CK(ctx, dcoef.ensure(t));
        NEO_CK(ctx, du.ensure(m));
        NEO_CK(ctx, cudaMemcpyAsync(dw.p, w.data(), nq * 16, cudaMemcpyHostToDevice, ctx->stream));
        NEO_CK(ctx, cudaMemcpyAsync(dcoef.p, coef.data(), t * 16, cudaMemcpyHostToDevice, ctx->stream));
        if (o->fast && (k - 1) * NEO_D / 2 <= EU_MAX_PAIRS) {  // ternary digits (checked above)
            const uint32_t cb = (uint32_t)ceil_div(m, 256);
            NEO_CK(ctx, o->ws_upart.ensure((size_t)EU_SPLIT * m));
            NEO_CK(ctx, o->ws_uticket.ensure(cb));
            NEO_CK(ctx, cudaMemsetAsync(o->ws_uticket.p, 0, cb * sizeof(unsigned int), ctx->stream));
            eval_u_pair_kernel<<<dim3(cb, EU_SPLIT), 256, 0, ctx->stream>>>(o->Z, m, k, dw.p, o->ws_upart.p,
                                                                         o->ws_uticket.p, du.p);
        } else {
            eval_u_kernel<<<ceil_div(m, 256), 256, 0, ctx->stream>>>(o->Z, m, k, dw.p, du.p);
        }
        NEO_LAUNCHED(ctx);
        DevBuf<uint8_t>& isid = o->ws_isid;
        NEO_CK(ctx, isid.ensure(t));
        NEO_CK(ctx, cudaMemcpyAsync(isid.p, o->ccs->is_identity.data(), t, cudaMemcpyHostToDevice, ctx->stream));
        DevBuf<uint64_t>& nnzoff = o->ws_nnzoff;
        NEO_CK(ctx, nnzoff.ensure(t + 1));
        NEO_CK(ctx, cudaMemcpyAsync(nnzoff.p, o->ccs->nnz_off.data(), (t + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
        eval_tbl_kernel<<<ceil_div(n_pad, 256), 256, 0, ctx->stream>>>(
            o->ccs->csr_ptr.p, o->ccs->csr_col.p, o->ccs->csr_val.p, nnzoff.p, isid.p, t, desc->n, desc->m, du.p,
            dcoef.p, n_pad, S + (size_t)o->idx_eval * n_pad);
        NEO_LAUNCHED(ctx);
        NEO_CK(ctx, ctx_sync(ctx));
    }
    // streamed rounds and the materialised NC table
    o->J = (int)std::min<uint32_t>(JMAX, ell_n - 1);
    if ((uint32_t)o->J < ell_n - 1) {
        uint64_t LJ = n_pad >> o->J;
        NEO_CK(ctx, o->nc[0].ensure((size_t)nq * LJ));
        NEO_CK(ctx, o->nc[1].ensure((size_t)nq * LJ / 2 + 1));
    }
    NEO_CK(ctx, o->eqw.ensure(1 << JMAX));
    NEO_CK(ctx, o->d_chals.ensure(o->ell_n ? o->ell_n : 1));
    uint64_t max_blocks = (uint64_t)ceil_div(n_pad / 2, RT) * nq + 16;
    NEO_CK(ctx, o->partials.ensure(max_blocks * (o->deg_max + 1)));
    NEO_CK(ctx, o->coeffs.ensure(MAX_DEG + 1));
    NEO_CK(ctx, o->ys.ensure(16));
    if (o->fast) {  // the pattern-histogram row rounds
        int rc2 = fast_setup(o);
        if (rc2) return rc2;
    }
    return NEO_OK;
}

// Grid of the NC blocks at round j >= 3: (pair, q chunk) threads, enough to
// fill the GPU about twice when the pairs alone do not.
static void fast_nc_grid(const neo_gpu_ccs_oracle* o, uint32_t j, uint32_t* n_chunk, uint32_t* q_chunk,
                         uint32_t* blocks) {
    const uint32_t nq = o->k * NEO_D;
    const uint64_t pairs = o->n_pad >> (j + 1);
    const uint64_t target = pairs < o->late_pairs ? o->late_threads : o->nc_threads;
    const uint32_t nc = (uint32_t)std::min<uint64_t>(nq, std::max<uint64_t>(1, (target + pairs - 1) / pairs));
    *q_chunk = (nq + nc - 1) / nc;
    *n_chunk = (nq + *q_chunk - 1) / *q_chunk;
    *blocks = (uint32_t)ceil_div(pairs * *n_chunk, FR);
}

static int fast_setup(neo_gpu_ccs_oracle* o) {
    neo_gpu_ctx* ctx = o->ctx;
    // launch choices: defaults, the tuned table of this shape (tune.cu), then
    // environment overrides
    o->compact_q = 8;
    o->nc_threads = 148ull * 2 * 256;
    o->hist_items = 16384;
    CcsTune tn;
    if (tune_lookup(o->ell_n, o->k, &tn)) {
        o->nc_threads = std::max<uint64_t>(1, tn.nc_threads);
        o->compact_q = tn.compact_q;
        o->hist_items = std::max<uint32_t>(1, tn.hist_items);
    }
    if (const char* e = getenv("NEO_TUNE_CCS_COMPACT_Q")) o->compact_q = (uint32_t)strtoul(e, nullptr, 10);
    if (const char* e = getenv("NEO_TUNE_CCS_NC_THREADS")) o->nc_threads = std::max<uint64_t>(1, strtoull(e, nullptr, 10));
    if (const char* e = getenv("NEO_TUNE_CCS_LATE_PAIRS")) o->late_pairs = strtoull(e, nullptr, 10);
    if (const char* e = getenv("NEO_TUNE_CCS_LATE_THREADS")) o->late_threads = std::max<uint64_t>(1, strtoull(e, nullptr, 10));
    const uint32_t ell = o->ell_n, nq = o->k * NEO_D;
    // E_j = chi of beta_r[j+1..ell) for every row round (beta_r is in ws_bits[0..ell))
    NEO_CK(ctx, o->E_all.ensure(o->n_pad));
    if (int rc = launch_suffix_chi_tables(ctx, o->ws_bits.p, ell, o->E_all.p)) return rc;
    // histogram grid: a thread per 8-row block, q chunks so that ~2 blocks per SM
    // split histograms (even / odd 8-row blocks) when round 3 exists
    const uint32_t n_t8 = (uint32_t)(o->n_pad >> 3);
    o->hist_split = ell >= 4;
    const uint32_t nz = o->hist_split ? 2 : 1;
    o->hist_gx = (uint32_t)ceil_div(n_t8 / nz, HIST_T);
    // one wave of 2 blocks per SM when it fits, but at least ~16k items per
    // block: a block zeroes, fills and writes out a 105 KB histogram
    const uint64_t items = (uint64_t)nq * n_t8;
    uint32_t gy = std::max<uint32_t>(1, 296 / (o->hist_gx * nz));
    gy = std::min<uint32_t>(gy, std::max<uint64_t>(1, items / ((uint64_t)o->hist_gx * nz * o->hist_items)));
    o->hist_qc = std::max<uint32_t>(1, std::min<uint32_t>(HIST_MAX_Q, (nq + gy - 1) / gy));
    o->hist_gy = (nq + o->hist_qc - 1) / o->hist_qc;
    NEO_CK(ctx, o->hist_part.ensure((size_t)nz * o->hist_gx * o->hist_gy * NPAT * HIST_LIMBS));
    NEO_CK(ctx, o->hist64.ensure((size_t)nz * NPAT * HIST_LIMBS));
    NEO_CK(ctx, o->ticket.ensure(1));
    NEO_CK(ctx, o->Cs.ensure(ell));
    NEO_CK(ctx, cudaMemsetAsync(o->ticket.p, 0, 4, ctx->stream));
    // partial records: the largest round
    uint64_t recs = 0;
    for (uint32_t j = 0; j < ell; j++) {
        uint64_t r = ceil_div(o->n_pad >> (j + 1), FR);
        if (j <= 3) r += ceil_div(NPAT, FR);
        if (j >= 3) {
            uint32_t nc, qc, blocks;
            fast_nc_grid(o, j, &nc, &qc, &blocks);
            r += blocks;
        }
        recs = std::max<uint64_t>(recs, r);
    }
    NEO_CK(ctx, o->partials.ensure(recs * REC));
    static SmemLimit hist_smem;
    NEO_CK(ctx, hist_smem.at_least(ccs_hist_kernel, (size_t)NPAT * HIST_LIMBS * 4 + HIST_MAX_Q * sizeof(K)));
    return NEO_OK;
}

// One row round on the ternary-digit path (one launch; round 0 first builds
// the pattern histogram); leaves deg_max + 1 coefficients in coeffs_dst
// (device).  d_chals must hold r_0..r_{j-1}.
static int fast_round_launch(neo_gpu_ccs_oracle* o, K* coeffs_dst) {
    neo_gpu_ctx* ctx = o->ctx;
    const uint32_t j = o->round_idx, ell = o->ell_n, nq = o->k * NEO_D;
    const bool last = j + 1 == ell;
    if (j == 0) {
        HistArgs h{};
        h.Z = o->Z;
        h.m = o->m;
        h.nq = nq;
        h.n_t8 = (uint32_t)(o->n_pad >> 3);
        h.q_chunk = o->hist_qc;
        h.wg = o->wg.p;
        const uint32_t jw = o->hist_split ? 3 : 2;  // E_3 per 16-row block, or E_2 per 8-row block
        h.Ew = o->E_all.p + (o->n_pad - (o->n_pad >> jw));
        h.split = o->hist_split;
        h.partial = o->hist_part.p;
        const uint32_t nz = o->hist_split ? 2 : 1;
        const size_t smem = (size_t)NPAT * HIST_LIMBS * 4 + (size_t)o->hist_qc * sizeof(K);
        ccs_hist_kernel<<<dim3(o->hist_gx, o->hist_gy, nz), HIST_T, smem, ctx->stream>>>(h);
        NEO_LAUNCHED(ctx);
        NEO_CK(ctx, cudaMemsetAsync(o->hist64.p, 0, (size_t)nz * NPAT * HIST_LIMBS * 8, ctx->stream));
        const uint32_t nblk = o->hist_gx * o->hist_gy;
        ccs_hist_sum_kernel<<<dim3((uint32_t)ceil_div(NPAT * HIST_LIMBS, 256), (uint32_t)ceil_div(nblk, HIST_SUM_SLICE), nz),
                              256, 0, ctx->stream>>>(o->hist_part.p, nblk,
                                                     reinterpret_cast<unsigned long long*>(o->hist64.p));
        NEO_LAUNCHED(ctx);
    }
    FastRoundArgs a{};
    a.j = (int)j;
    a.n_mom = j <= 3 ? (uint32_t)ceil_div(NPAT, FR) : 0;  // moments (rounds 0..2), separable terms (round 3)
    a.H64 = reinterpret_cast<const unsigned long long*>(o->hist64.p);
    a.split = o->hist_split;
    a.beta1 = o->beta_r[1];
    a.beta2 = o->beta_r[2];
    if (o->hist_split) a.beta3 = o->beta_r[3];
    if (j == 0) {
        a.small_in = o->small[0].p;
        a.small_len_in = o->n_pad;
        a.fold = 0;
    } else {
        a.small_in = o->small[o->small_cur].p;
        a.small_len_in = o->n_pad >> (j - 1);
        a.fold = 1;
        a.r = o->row_chals[j - 1];
        a.small_out = last ? nullptr : o->small[o->small_cur ^ 1].p;
        a.small_len_out = o->n_pad >> j;
    }
    a.n_small_tab = o->n_small;
    a.idx_eqrin = o->idx_eqrin;
    a.idx_eval = o->idx_eval;
    a.f = o->f;
    a.fdeg = o->deg_max - 1;
    a.E = o->E_all.p + (o->n_pad - (o->n_pad >> j));
    a.pairs = o->n_pad >> (j + 1);
    a.n_small = (uint32_t)ceil_div(a.pairs, FR);
    a.chals = o->d_chals.p;
    a.Z = o->Z;
    a.m = o->m;
    a.wg = o->wg.p;
    a.nq = nq;
    uint32_t nc_blocks = 0;
    if (j >= 3) {
        fast_nc_grid(o, j, &a.n_chunk, &a.q_chunk, &nc_blocks);
        if (j == 4 && !last) {
            a.nc_out = o->nc[0].p;
            a.nc_len_out = o->n_pad >> 4;
            o->nc_cur = 0;
        } else if (j >= 5) {
            a.nc_in = o->nc[o->nc_cur].p;
            a.nc_len_in = o->n_pad >> (j - 1);
            if (!last) {
                a.nc_out = o->nc[o->nc_cur ^ 1].p;
                a.nc_len_out = o->n_pad >> j;
            }
        }
    }
    a.partials = o->partials.p;
    a.ticket = o->ticket.p;
    a.ncoef = o->deg_max + 1;
    for (uint32_t i = 0; i < ell && i < 32; i++) a.beta[i] = o->beta_r[i];
    a.gamma_to_k = o->gamma_to_k;
    a.Cs = o->Cs.p;
    a.coeffs_out = coeffs_dst;
    const uint32_t blocks = a.n_mom + a.n_small + nc_blocks;
    const size_t wsm = j >= 3 ? (size_t)nq * sizeof(K) : 0;
    // a thread that evaluates few q runs its K products out of line (compact code)
    const bool compact = j >= 3 && a.q_chunk < o->compact_q;
    if (j <= 2) ccs_fast_round_kernel<0, true><<<blocks, FR, 0, ctx->stream>>>(a);
    else if (j == 3) {
        if (compact) ccs_fast_round_kernel<3, true><<<blocks, FR, wsm, ctx->stream>>>(a);
        else ccs_fast_round_kernel<3, false><<<blocks, FR, wsm, ctx->stream>>>(a);
    } else if (j == 4) {
        if (compact) ccs_fast_round_kernel<4, true><<<blocks, FR, wsm, ctx->stream>>>(a);
        else ccs_fast_round_kernel<4, false><<<blocks, FR, wsm, ctx->stream>>>(a);
    } else {
        if (compact) ccs_fast_round_kernel<5, true><<<blocks, FR, wsm, ctx->stream>>>(a);
        else ccs_fast_round_kernel<5, false><<<blocks, FR, wsm, ctx->stream>>>(a);
    }
    NEO_LAUNCHED(ctx);
    if (j > 0 && !last) o->small_cur ^= 1;
    if (j >= 5 && !last) o->nc_cur ^= 1;
    return NEO_OK;
}

// Launches row round j = round_idx (folding the previous challenge in) and
// leaves its deg_max + 1 coefficients in coeffs_dst (device); no host sync.
// d_chals must hold the row challenges of the rounds already bound.
static int row_round_launch(neo_gpu_ccs_oracle* o, K* coeffs_dst) {
    if (o->fast) return fast_round_launch(o, coeffs_dst);
    neo_gpu_ctx* ctx = o->ctx;
    const uint32_t j = o->round_idx;
    const uint32_t nq = o->k * NEO_D;
    RoundArgs a{};
    a.pairs = o->n_pad >> (j + 1);
    a.n_small = o->n_small;
    a.n_fvar = o->n_fvar;
    a.idx_eqrin = o->idx_eqrin;
    a.idx_eval = o->idx_eval;
    a.gamma_to_k = o->gamma_to_k;
    a.f = o->f;
    a.deg_max = o->deg_max;
    a.wg = o->wg.p;
    a.nq = (int)nq;
    a.Z = o->Z;
    a.m = o->m;
    const bool last = j + 1 == o->ell_n;
    // small tables
    if (j == 0) {
        a.small_in = o->small[0].p;
        a.small_len_in = o->n_pad;
        a.fold = 0;
        a.small_out = nullptr;
    } else {
        a.small_in = o->small[o->small_cur].p;
        a.small_len_in = o->n_pad >> (j - 1);
        a.fold = 1;
        a.r = o->row_chals[j - 1];
        a.small_out = last ? nullptr : o->small[o->small_cur ^ 1].p;
        a.small_len_out = o->n_pad >> j;
    }
    // NC source
    const int J = o->J;
    if ((int)j <= J) {
        if (j > 0) {
            // χ of the bound prefix r_0..r_{j-1}
            int rc = launch_chi_table(ctx, o->d_chals.p, j, o->eqw.p);
            if (rc) return rc;
        }
        a.eqw = o->eqw.p;
        if ((int)j == J && !last) {
            a.nc_out = o->nc[0].p;
            a.nc_len_out = o->n_pad >> j;
            o->nc_cur = 0;
        }
    } else {
        a.nc_in = o->nc[o->nc_cur].p;
        a.nc_len_in = o->n_pad >> (j - 1);
        a.r = o->row_chals[j - 1];
        if (!last) {
            a.nc_out = o->nc[o->nc_cur ^ 1].p;
            a.nc_len_out = o->n_pad >> j;
        }
    }
    // grid: x over pairs, y over q-chunks so that the GPU is filled
    unsigned gx = ceil_div(a.pairs, RT);
    unsigned target = 148 * 6;
    unsigned gy = std::min<unsigned>(nq, std::max<unsigned>(1, (target + gx - 1) / gx));
    int qpb = (int)ceil_div(nq, gy);
    if (qpb > 1024) qpb = 1024;
    gy = ceil_div(nq, qpb);
    a.q_per_block = qpb;
    a.partials = o->partials.p;
    dim3 grid(gx, gy);
    switch ((int)j <= J ? (int)j : JMAX + 1) {
        case 0: ccs_round_kernel<0><<<grid, RT, 0, ctx->stream>>>(a); break;
        case 1: ccs_round_kernel<1><<<grid, RT, 0, ctx->stream>>>(a); break;
        case 2: ccs_round_kernel<2><<<grid, RT, 0, ctx->stream>>>(a); break;
        case 3: ccs_round_kernel<3><<<grid, RT, 0, ctx->stream>>>(a); break;
        case 4: ccs_round_kernel<4><<<grid, RT, 0, ctx->stream>>>(a); break;
        default: ccs_round_kernel<JMAX + 1><<<grid, RT, 0, ctx->stream>>>(a); break;
    }
    NEO_LAUNCHED(ctx);
    if (j > 0 && !last) o->small_cur ^= 1;
    if ((int)j > J && !last) o->nc_cur ^= 1;
    // reduce
    EvalArgs e{};
    e.partials = o->partials.p;
    e.nblocks = gx * gy;
    e.ncoef = o->deg_max + 1;
    e.nx = 0;
    e.coeffs_out = coeffs_dst;
    e.ys_out = o->ys.p;
    reduce_eval_kernel<<<1, 256, 0, ctx->stream>>>(e);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}

static int row_round(neo_gpu_ccs_oracle* o) {
    neo_gpu_ctx* ctx = o->ctx;
    const uint32_t j = o->round_idx;
    if (j > 0 && ((int)j <= o->J || o->fast))
        NEO_CK(ctx, cudaMemcpyAsync(o->d_chals.p, o->row_chals.data(), j * sizeof(K), cudaMemcpyHostToDevice,
                                    ctx->stream));
    int rc = row_round_launch(o, o->coeffs.p);
    if (rc) return rc;
    o->h_coeffs.resize(o->deg_max + 1);
    NEO_CK(ctx, ctx_d2h(ctx, o->h_coeffs.data(), o->coeffs.p, (o->deg_max + 1) * 16));
    NEO_CK(ctx, ctx_sync(ctx));
    o->coeffs_valid = true;
    return NEO_OK;
}

// Enqueues the current row round with its coefficients (deg_max + 1 K values)
// written to d_dst on the device and no host sync (the batched sum-check
// launches every claim of a round, then copies all values back at once).
int ccs_oracle_round_launch(neo_gpu_ccs_oracle* o, K* d_dst, uint32_t* ncoef) {
    neo_gpu_ctx* ctx = o->ctx;
    const uint32_t j = o->round_idx;
    if (j >= o->ell_n) return ctx->fail(NEO_ERR_ARG, "ccs round launch: not a row round");
    if (j > 0 && ((int)j <= o->J || o->fast)) {
        NEO_CK(ctx, o->h_chals.ensure(o->ell_n));
        memcpy(o->h_chals.p, o->row_chals.data(), j * sizeof(K));
        NEO_CK(ctx, cudaMemcpyAsync(o->d_chals.p, o->h_chals.p, j * sizeof(K), cudaMemcpyHostToDevice, ctx->stream));
    }
    int rc = row_round_launch(o, d_dst);
    if (rc) return rc;
    *ncoef = (uint32_t)o->deg_max + 1;
    return NEO_OK;
}

// The coefficients of the round just launched, read back by the caller.
void ccs_oracle_round_set(neo_gpu_ccs_oracle* o, const K* coeffs) {
    o->h_coeffs.assign(coeffs, coeffs + o->deg_max + 1);
    o->coeffs_valid = true;
}

static int ajtai_precompute(neo_gpu_ccs_oracle* o) {
    neo_gpu_ctx* ctx = o->ctx;
    NEO_CK(ctx, o->chi_r.ensure(o->n_pad));
    NEO_CK(ctx, o->vj.ensure((size_t)o->t * o->m));
    NEO_CK(ctx, o->y_eval.ensure((size_t)o->k * o->t * NEO_D));
    NEO_CK(ctx, o->y_sc.ensure((size_t)o->k * o->t));
    DevBuf<K>& dbits = o->ws_bits;
    NEO_CK(ctx, dbits.ensure(2 * o->ell_n));
    NEO_CK(ctx, cudaMemcpyAsync(dbits.p, o->row_chals.data(), o->ell_n * 16, cudaMemcpyHostToDevice, ctx->stream));
    int rc = launch_chi_table(ctx, dbits.p, o->ell_n, o->chi_r.p);
    if (rc) return rc;
    rc = launch_me_y(ctx, *o->ccs, o->Z, o->k, o->m, o->chi_r.p, o->ell_n, o->b, o->vj.p, o->y_eval.p, o->y_sc.p,
                     o->fast);  // fast: every digit checked ternary at creation
    if (rc) return rc;
    NEO_CK(ctx, ctx_sync(ctx));
    o->have_pre = true;
    return NEO_OK;
}

static int ajtai_round(neo_gpu_ccs_oracle* o, const uint64_t* xs, uint32_t nx, uint64_t* ys) {
    neo_gpu_ctx* ctx = o->ctx;
    if (!o->have_pre) {
        int rc = ajtai_precompute(o);
        if (rc) return rc;
    }
    if (nx > 16 || o->ell_n > 32 || o->ell_d > 8 || o->k * (1 + o->t) > 160)
        return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_oracle: ajtai phase size limits");
    AjtaiArgs a{};
    a.k = (int)o->k; a.t = (int)o->t; a.ell_d = (int)o->ell_d; a.ell_n = (int)o->ell_n;
    a.j = (int)(o->round_idx - o->ell_n);
    a.nx = (int)nx;
    a.has_inputs = o->has_inputs;
    for (uint32_t i = 0; i < nx; i++) a.xs[i] = gl::kmk(gl::canon(xs[2 * i]), gl::canon(xs[2 * i + 1]));
    for (uint32_t i = 0; i < o->ell_d; i++) { a.alpha[i] = o->alpha[i]; a.beta_a[i] = o->beta_a[i]; }
    for (size_t i = 0; i < o->ajtai_chals.size(); i++) a.ajtai_chals[i] = o->ajtai_chals[i];
    for (uint32_t i = 0; i < o->ell_n; i++) {
        a.beta_r[i] = o->beta_r[i];
        a.row_chals[i] = o->row_chals[i];
        if (o->has_inputs) a.r_in[i] = o->r_in[i];
    }
    a.gamma = o->gamma;
    a.f = o->f;
    for (int v = 0; v < o->n_fvar; v++) a.fvar_j[v] = o->fvar_j[v];
    a.y = o->y_eval.p;
    a.ysc = o->y_sc.p;
    a.ys_out = o->ys.p;
    size_t smem = ((size_t)o->k * (1 + o->t) * NEO_D + (size_t)nx * o->k) * sizeof(K);
    static SmemLimit limit;
    NEO_CK(ctx, limit.at_least(ajtai_round_kernel, smem));
    ajtai_round_kernel<<<1, 512, smem, ctx->stream>>>(a);
    NEO_LAUNCHED(ctx);
    NEO_CK(ctx, ctx_d2h(ctx, ys, o->ys.p, nx * 16));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}

static int neo_gpu_ccs_oracle_evals_impl_abi(neo_gpu_ccs_oracle* o, const uint64_t* xs, uint32_t nx, uint64_t* ys) {
    if (!o) return NEO_ERR_ARG;
    neo_gpu_ctx* ctx = o->ctx;
    if (!xs || !ys || nx == 0 || nx > 16) return ctx->fail(NEO_ERR_ARG, "evals: bad args");
    if (o->round_idx >= o->ell_n + o->ell_d) return ctx->fail(NEO_ERR_ARG, "evals: all rounds done");
    cudaSetDevice(ctx->device);
    if (o->round_idx < o->ell_n) {
        if (!o->coeffs_valid) {
            int rc = row_round(o);
            if (rc) return rc;
        }
        // Horner at each x (sumcheck.rs:48-60)
        for (uint32_t i = 0; i < nx; i++) {
            K x = gl::kmk(gl::canon(xs[2 * i]), gl::canon(xs[2 * i + 1]));
            K r = o->h_coeffs.back();
            for (int d = (int)o->h_coeffs.size() - 2; d >= 0; d--) r = gl::kadd(gl::kmul(r, x), o->h_coeffs[d]);
            ys[2 * i] = r.re;
            ys[2 * i + 1] = r.im;
        }
        return NEO_OK;
    }
    return ajtai_round(o, xs, nx, ys);
}
extern "C" int neo_gpu_ccs_oracle_evals(neo_gpu_ccs_oracle* o, const uint64_t* xs, uint32_t nx, uint64_t* ys) { NEO_ABI_GUARD(neo_gpu_ccs_oracle_evals_impl_abi(o, xs, nx, ys)) }

static int neo_gpu_ccs_oracle_fold_impl_abi(neo_gpu_ccs_oracle* o, const uint64_t* r) {
    if (!o) return NEO_ERR_ARG;
    if (!r) return o->ctx->fail(NEO_ERR_ARG, "fold: null r");
    K rr = gl::kmk(gl::canon(r[0]), gl::canon(r[1]));
    if (o->round_idx < o->ell_n) {
        o->row_chals.push_back(rr);
        o->coeffs_valid = false;
    } else if (o->round_idx < o->ell_n + o->ell_d) {
        o->ajtai_chals.push_back(rr);
    } else {
        return o->ctx->fail(NEO_ERR_ARG, "fold: all rounds done");
    }
    o->round_idx++;
    return NEO_OK;
}
extern "C" int neo_gpu_ccs_oracle_fold(neo_gpu_ccs_oracle* o, const uint64_t* r) { NEO_ABI_GUARD(neo_gpu_ccs_oracle_fold_impl_abi(o, r)) }

static int neo_gpu_ccs_oracle_row_rounds_device_impl_abi(neo_gpu_ccs_oracle* o, const uint64_t* chals, uint32_t n,
                                                    uint64_t* d_coeffs) {
    if (!o) return NEO_ERR_ARG;
    neo_gpu_ctx* ctx = o->ctx;
    if (!chals || !d_coeffs || n == 0) return ctx->fail(NEO_ERR_ARG, "row_rounds_device: bad args");
    if (o->round_idx + n > o->ell_n) return ctx->fail(NEO_ERR_ARG, "row_rounds_device: beyond the row rounds");
    cudaSetDevice(ctx->device);
    const uint32_t j0 = o->round_idx;
    for (uint32_t i = 0; i < n; i++) o->row_chals.push_back(gl::kmk(gl::canon(chals[2 * i]), gl::canon(chals[2 * i + 1])));
    // every challenge of the sequence goes up once; round j reads only the first j
    NEO_CK(ctx, cudaMemcpyAsync(o->d_chals.p, o->row_chals.data(), (j0 + n) * sizeof(K), cudaMemcpyHostToDevice,
                                ctx->stream));
    // rounds are written at stride d_sc + 1; coefficients above deg_max are zero
    const uint32_t ncoef = o->d_sc + 1;
    if ((uint32_t)o->deg_max > o->d_sc) return ctx->fail(NEO_ERR_INVARIANT, "row_rounds_device: degree above d_sc");
    NEO_CK(ctx, cudaMemsetAsync(d_coeffs, 0, (size_t)n * ncoef * sizeof(K), ctx->stream));
    for (uint32_t i = 0; i < n; i++) {
        int rc = row_round_launch(o, reinterpret_cast<K*>(d_coeffs) + (size_t)i * ncoef);
        if (rc) return rc;
        o->round_idx++;
    }
    o->coeffs_valid = false;
    return NEO_OK;
}
extern "C" int neo_gpu_ccs_oracle_row_rounds_device(neo_gpu_ccs_oracle* o, const uint64_t* chals, uint32_t n,
                                                    uint64_t* d_coeffs) { NEO_ABI_GUARD(neo_gpu_ccs_oracle_row_rounds_device_impl_abi(o, chals, n, d_coeffs)) }

extern "C" uint32_t neo_gpu_ccs_oracle_num_rounds(const neo_gpu_ccs_oracle* o) { return o ? o->ell_n + o->ell_d : 0; }
extern "C" uint32_t neo_gpu_ccs_oracle_degree_bound(const neo_gpu_ccs_oracle* o) { return o ? o->d_sc : 0; }

static int neo_gpu_ccs_oracle_me_outputs_impl_abi(neo_gpu_ccs_oracle* o, uint64_t* y, uint64_t* y_scalars) {
    if (!o) return NEO_ERR_ARG;
    neo_gpu_ctx* ctx = o->ctx;
    if (!y || !y_scalars) return ctx->fail(NEO_ERR_ARG, "me_outputs: null output");
    if (o->row_chals.size() != o->ell_n) return ctx->fail(NEO_ERR_ARG, "me_outputs: row challenges not finalized");
    cudaSetDevice(ctx->device);
    if (!o->have_pre) {
        int rc = ajtai_precompute(o);
        if (rc) return rc;
    }
    NEO_CK(ctx, ctx_d2h(ctx, y, o->y_eval.p, o->y_eval.bytes()));
    NEO_CK(ctx, ctx_d2h(ctx, y_scalars, o->y_sc.p, o->y_sc.bytes()));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_ccs_oracle_me_outputs(neo_gpu_ccs_oracle* o, uint64_t* y, uint64_t* y_scalars) { NEO_ABI_GUARD(neo_gpu_ccs_oracle_me_outputs_impl_abi(o, y, y_scalars)) }

static int neo_gpu_ccs_oracle_destroy_impl_abi(neo_gpu_ccs_oracle* o) {
    if (!o) return NEO_ERR_ARG;
    cudaSetDevice(o->ctx->device);
    cudaStreamSynchronize(o->ctx->stream);
    delete o;
    return NEO_OK;
}
extern "C" int neo_gpu_ccs_oracle_destroy(neo_gpu_ccs_oracle* o) { NEO_ABI_GUARD(neo_gpu_ccs_oracle_destroy_impl_abi(o)) }

// device view of v_j = M_j^T chi_r' for the fold step (child ME claims reuse it)
int ccs_oracle_dev_vj(neo_gpu_ccs_oracle* o, const K** vj) {
    if (o->row_chals.size() != o->ell_n) return o->ctx->fail(NEO_ERR_ARG, "dev_vj: row phase not finished");
    if (!o->have_pre) {
        int rc = ajtai_precompute(o);
        if (rc) return rc;
    }
    *vj = o->vj.p;
    return NEO_OK;
}

// ---------------------------------------------------------------------------
// Autotuner of the ternary-digit row rounds (tune.cu): every candidate launch
// choice runs the whole row-round sequence of the caller's CCS and witness
// digits (random challenges); the fastest is recorded for (ell_n, k).
// ---------------------------------------------------------------------------
static uint64_t tune_mix(uint64_t& s) {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return gl::canon(z ^ (z >> 31));
}

static int neo_gpu_ccs_autotune_impl_abi(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, const int8_t* Z, uint32_t k,
                                         uint32_t reps, uint64_t* best3) {
    if (!ctx) return NEO_ERR_ARG;
    if (!desc || !Z || !best3 || k == 0 || reps == 0) return ctx->fail(NEO_ERR_ARG, "ccs_autotune: bad args");
    uint32_t ell_n = 0;
    while ((1u << ell_n) < desc->n) ell_n++;
    if (desc->n != desc->m || (1u << ell_n) != desc->n || ell_n < 3)
        return ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_autotune: needs n == m == 2^ell, ell >= 3");
    NEO_CK(ctx, cudaSetDevice(ctx->device));
    const uint32_t ell_d = 6, d_sc = 6;
    uint64_t seed = 0x4E454F54554E45ull;
    auto rk = [&](size_t n) {
        std::vector<K> v(n);
        for (auto& x : v) x = gl::kmk(tune_mix(seed), tune_mix(seed));
        return v;
    };
    std::vector<K> al = rk(ell_d), ba = rk(ell_d), br = rk(ell_n), ri = rk(ell_n), g = rk(1), ch = rk(ell_n);
    auto* o = new neo_gpu_ccs_oracle();
    std::unique_ptr<neo_gpu_ccs_oracle> guard(o);
    int rc = dev_ccs_upload(ctx, desc, o->own_ccs);
    if (rc) return rc;
    o->ccs = &o->own_ccs;
    NEO_CK(ctx, o->own_Z.alloc((size_t)k * NEO_D * desc->m));
    NEO_CK(ctx, cudaMemcpyAsync(o->own_Z.p, Z, o->own_Z.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    DevBuf<K> coeffs;
    NEO_CK(ctx, coeffs.ensure((size_t)ell_n * (MAX_DEG + 1)));
    cudaEvent_t e0, e1;
    NEO_CK(ctx, cudaEventCreate(&e0));
    NEO_CK(ctx, cudaEventCreate(&e1));
    const uint64_t wave = 148ull * 2 * FR;
    const uint64_t nts[3] = {wave / 2, wave, 2 * wave};
    const uint32_t cqs[3] = {0, 8, 64}, his[3] = {8192, 16384, 65536};
    CcsTune best{wave, 8, 16384};
    float best_ms = 1e30f;
    for (uint64_t nt : nts)
        for (uint32_t cq : cqs)
            for (uint32_t hi : his) {
                CcsTune cand{nt, cq, hi};
                float cand_ms = 1e30f;
                for (uint32_t rep = 0; rep < reps + 1 && rc == 0; rep++) {
                    tune_force(&cand);
                    rc = oracle_init(ctx, o, o->own_Z.p, k, 2, al.data(), ba.data(), br.data(), g[0], ri.data(), ell_d,
                                     ell_n, d_sc);
                    tune_force(nullptr);
                    if (rc) break;
                    if (!o->fast) {
                        rc = ctx->fail(NEO_ERR_UNSUPPORTED, "ccs_autotune: digits are not ternary");
                        break;
                    }
                    o->row_chals.assign(ch.begin(), ch.end());
                    NEO_CK(ctx, cudaMemcpyAsync(o->d_chals.p, ch.data(), ell_n * sizeof(K), cudaMemcpyHostToDevice,
                                                ctx->stream));
                    NEO_CK(ctx, cudaEventRecord(e0, ctx->stream));
                    for (uint32_t j = 0; j < ell_n && rc == 0; j++) {
                        o->round_idx = j;
                        rc = row_round_launch(o, coeffs.p + (size_t)j * (MAX_DEG + 1));
                    }
                    NEO_CK(ctx, cudaEventRecord(e1, ctx->stream));
                    NEO_CK(ctx, cudaEventSynchronize(e1));
                    float ms = 0;
                    NEO_CK(ctx, cudaEventElapsedTime(&ms, e0, e1));
                    if (rep > 0 && ms < cand_ms) cand_ms = ms;  // the first run warms up
                }
                if (rc) break;
                if (cand_ms < best_ms) {
                    best_ms = cand_ms;
                    best = cand;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    tune_store(ell_n, k, best);
    best3[0] = best.nc_threads;
    best3[1] = best.compact_q;
    best3[2] = best.hist_items;
    return NEO_OK;
}
extern "C" int neo_gpu_ccs_autotune(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, const int8_t* Z, uint32_t k,
                                    uint32_t reps, uint64_t* best3) {
    NEO_ABI_GUARD(neo_gpu_ccs_autotune_impl_abi(ctx, desc, Z, k, reps, best3))
}
