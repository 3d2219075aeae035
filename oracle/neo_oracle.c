/*
 * neo_oracle.c -- CPU restatement of the Neo fold-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); the
 * product never links this file.  See neo_oracle.h for the parity status.
 * Citations are path:line within the reference project.
 */
#include "neo_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;
#define D OR_D
#define Q OR_Q
#define EPS 0xFFFFFFFFULL /* 2^64 mod q = 2^32 - 1 */

/* ------------------------------------------------------------------------ */
/* Fq: Goldilocks.  Reduction of a 128-bit product uses 2^64 = 2^32-1 and    */
/* 2^96 = -1 (mod q); a standard published identity for this prime.         */
/* ------------------------------------------------------------------------ */
static inline uint64_t fq_canon(uint64_t a) { return a >= Q ? a - Q : a; }
static inline uint64_t fq_add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    uint64_t c = (s < a);              /* carry => s + 2^64 = s + EPS (mod q) */
    s += c * EPS;
    /* s < 2^64 here because a,b < q */
    return fq_canon(s);
}
static inline uint64_t fq_sub(uint64_t a, uint64_t b) {
    return a >= b ? a - b : a + (Q - b);
}
static inline uint64_t fq_neg(uint64_t a) { return a == 0 ? 0 : Q - a; }
static inline uint64_t fq_reduce128(u128 x) {
    uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
    uint64_t hi_hi = hi >> 32, hi_lo = hi & EPS;
    uint64_t t0 = lo - hi_hi;
    if (lo < hi_hi) t0 -= EPS;         /* borrow: -2^64 = -EPS */
    uint64_t t1 = hi_lo * EPS;         /* < 2^64 */
    uint64_t s = t0 + t1;
    if (s < t0) s += EPS;              /* carry */
    return fq_canon(s);
}
static inline uint64_t fq_mul(uint64_t a, uint64_t b) { return fq_reduce128((u128)a * b); }
static inline uint64_t fq_from_i64(int64_t v) { return v >= 0 ? (uint64_t)v : Q - (uint64_t)(-v); }
static uint64_t fq_pow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    while (e) { if (e & 1) r = fq_mul(r, a); a = fq_mul(a, a); e >>= 1; }
    return r;
}
static inline uint64_t fq_inv(uint64_t a) { return fq_pow(a, Q - 2); }

/* ------------------------------------------------------------------------ */
/* K = Fq[u]/(u^2 - 7)   (neo-math/src/field.rs:13; s_action.rs:65)          */
/* ------------------------------------------------------------------------ */
typedef struct { uint64_t re, im; } kq;
static const kq K0 = {0, 0};
static const kq K1 = {1, 0};
static inline kq kk(uint64_t re, uint64_t im) { kq r = {re, im}; return r; }
static inline kq kload(const uint64_t* p) { return kk(p[0], p[1]); }
static inline void kstore(uint64_t* p, kq a) { p[0] = a.re; p[1] = a.im; }
static inline kq kadd(kq a, kq b) { return kk(fq_add(a.re, b.re), fq_add(a.im, b.im)); }
static inline kq ksub(kq a, kq b) { return kk(fq_sub(a.re, b.re), fq_sub(a.im, b.im)); }
static inline kq kneg(kq a) { return kk(fq_neg(a.re), fq_neg(a.im)); }
static inline kq kmul(kq a, kq b) {
    uint64_t rr = fq_add(fq_mul(a.re, b.re), fq_mul(7, fq_mul(a.im, b.im)));
    uint64_t ii = fq_add(fq_mul(a.re, b.im), fq_mul(a.im, b.re));
    return kk(rr, ii);
}
static inline kq kscale(kq a, uint64_t s) { return kk(fq_mul(a.re, s), fq_mul(a.im, s)); }
static inline int keq(kq a, kq b) { return a.re == b.re && a.im == b.im; }
static inline int kiszero(kq a) { return a.re == 0 && a.im == 0; }
static inline kq kfq(uint64_t a) { return kk(a, 0); }
static kq kinv(kq a) {
    /* (a0 + a1 u)^{-1} = (a0 - a1 u) / (a0^2 - 7 a1^2) */
    uint64_t n = fq_sub(fq_mul(a.re, a.re), fq_mul(7, fq_mul(a.im, a.im)));
    uint64_t ni = fq_inv(n);
    return kk(fq_mul(a.re, ni), fq_mul(fq_neg(a.im), ni));
}

void or_fq_mul_batch(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out) {
    for (size_t i = 0; i < n; i++) out[i] = fq_mul(a[i], b[i]);
}
void or_k_mul_batch(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out) {
    for (size_t i = 0; i < n; i++) kstore(out + 2 * i, kmul(kload(a + 2 * i), kload(b + 2 * i)));
}
void or_k_inv_batch(const uint64_t* a, size_t n, uint64_t* out) {
    for (size_t i = 0; i < n; i++) kstore(out + 2 * i, kinv(kload(a + 2 * i)));
}

/* ------------------------------------------------------------------------ */
/* Rq schoolbook multiply mod Phi_81 = X^54 + X^27 + 1 (ring.rs:54-67,187-204)*/
/* ------------------------------------------------------------------------ */
static void reduce_mod_phi81(uint64_t* c /* [2D-1] */) {
    for (int i = 2 * D - 2; i >= D; i--) {
        uint64_t t = c[i];
        c[i] = 0;
        c[i - D] = fq_sub(c[i - D], t);
        int i27 = i - 27;
        if (i27 < D) {
            c[i27] = fq_sub(c[i27], t);
        } else {
            c[i27 - D] = fq_add(c[i27 - D], t);
            if (i27 - 27 < D) c[i27 - 27] = fq_add(c[i27 - 27], t);
        }
    }
}
void or_rq_mul(const uint64_t* a, const uint64_t* b, uint64_t* out) {
    uint64_t tmp[2 * D - 1];
    memset(tmp, 0, sizeof tmp);
    for (int i = 0; i < D; i++)
        for (int j = 0; j < D; j++) tmp[i + j] = fq_add(tmp[i + j], fq_mul(a[i], b[j]));
    reduce_mod_phi81(tmp);
    memcpy(out, tmp, D * sizeof(uint64_t));
}

/* rot_step for Phi_81 (commit.rs:46-54): column t -> t+1 */
static inline void rot_step(const uint64_t* cur, uint64_t* nxt) {
    uint64_t last = cur[D - 1];
    nxt[0] = fq_neg(last);
    for (int k = 1; k < D; k++) nxt[k] = cur[k - 1];
    nxt[27] = fq_sub(nxt[27], last);
}

/* commit_precomp_ct_row_major (commit.rs:679-744): c_i = sum_j rot(a_ij) Z[:,j].
   Digit masks in {-1,0,1} take the add/sub fast path of acc_mul_add_inplace
   (commit.rs:73-131); any other digit value multiplies. */
void or_commit_digits(const uint64_t* pp, int kappa, int64_t m, const int8_t* Z, uint64_t* out, int threads) {
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    (void)threads;
#endif
    for (int i = 0; i < kappa; i++) {
        uint64_t acc[D];
        memset(acc, 0, sizeof acc);
#ifdef _OPENMP
#pragma omp parallel num_threads(threads)
#endif
        {
            uint64_t lacc[D];
            uint64_t cols[D][D];
            memset(lacc, 0, sizeof lacc);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
            for (int64_t j = 0; j < m; j++) {
                const uint64_t* a = pp + ((size_t)i * m + j) * D;
                memcpy(cols[0], a, sizeof(uint64_t) * D);
                for (int t = 1; t < D; t++) rot_step(cols[t - 1], cols[t]);
                for (int t = 0; t < D; t++) {
                    int8_t z = Z[(size_t)t * m + j];
                    if (z == 0) continue;
                    if (z == 1) {
                        for (int r = 0; r < D; r++) lacc[r] = fq_add(lacc[r], cols[t][r]);
                    } else if (z == -1) {
                        for (int r = 0; r < D; r++) lacc[r] = fq_sub(lacc[r], cols[t][r]);
                    } else {
                        uint64_t s = fq_from_i64(z);
                        for (int r = 0; r < D; r++) lacc[r] = fq_add(lacc[r], fq_mul(cols[t][r], s));
                    }
                }
            }
#ifdef _OPENMP
#pragma omp critical
#endif
            for (int r = 0; r < D; r++) acc[r] = fq_add(acc[r], lacc[r]);
        }
        memcpy(out + (size_t)i * D, acc, sizeof acc);
    }
}

/* commit_masked_ct semantics over a general Fq matrix (commit.rs:512-553) */
void or_commit_fq(const uint64_t* pp, int kappa, int64_t m, const uint64_t* Z, uint64_t* out) {
    for (int i = 0; i < kappa; i++) {
        uint64_t acc[D], col[D], nxt[D];
        memset(acc, 0, sizeof acc);
        for (int64_t j = 0; j < m; j++) {
            memcpy(col, pp + ((size_t)i * m + j) * D, sizeof col);
            for (int t = 0; t < D; t++) {
                uint64_t mask = Z[(size_t)t * m + j];
                for (int r = 0; r < D; r++) acc[r] = fq_add(acc[r], fq_mul(col[r], mask));
                rot_step(col, nxt);
                memcpy(col, nxt, sizeof col);
            }
        }
        memcpy(out + (size_t)i * D, acc, sizeof acc);
    }
}

/* to_balanced_i64 (neo-ajtai/src/util.rs:19-29) */
static inline int64_t to_balanced_i64(uint64_t u) {
    const uint64_t half = (Q - 1) / 2;
    return u <= half ? (int64_t)u : -(int64_t)(Q - u);
}

/* decomp_b_row_major, b=2 Balanced (decomp.rs:118-158) */
void or_decomp_b2(const uint64_t* z, int64_t m, int8_t* Z) {
    for (int64_t c = 0; c < m; c++) {
        int64_t a = to_balanced_i64(z[c]);
        for (int row = 0; row < D; row++) {
            int64_t digit = (a & 1) == 0 ? 0 : (a >= 0 ? 1 : -1);
            Z[(size_t)row * m + c] = (int8_t)digit;
            a = (a - digit) >> 1;
        }
    }
}

/* recomposed_z_from_Z (paper_exact.rs:52-78), b=2 */
void or_recompose_b2(const int8_t* Z, int64_t m, uint64_t* z) {
    uint64_t pw[D];
    pw[0] = 1;
    for (int i = 1; i < D; i++) pw[i] = fq_mul(pw[i - 1], 2);
    for (int64_t c = 0; c < m; c++) {
        uint64_t acc = 0;
        for (int rho = 0; rho < D; rho++)
            acc = fq_add(acc, fq_mul(fq_from_i64(Z[(size_t)rho * m + c]), pw[rho]));
        z[c] = acc;
    }
}

/* ------------------------------------------------------------------------ */
/* RLC / DEC                                                                 */
/* ------------------------------------------------------------------------ */
/* rot_from_coeffs (common.rs:398-430): column j = cf(a X^j) */
void or_rot_matrix(const int8_t* a, uint64_t* out) {
    uint64_t col[D], nxt[D];
    for (int r = 0; r < D; r++) col[r] = fq_from_i64(a[r]);
    for (int j = 0; j < D; j++) {
        for (int r = 0; r < D; r++) out[r * D + j] = col[r];
        rot_step(col, nxt);
        memcpy(col, nxt, sizeof col);
    }
}

/* Z_mix = sum_i rho_i Z_i (rlc_reduction_optimized, optimized_engine/common.rs:1221-1379;
   left_mul_acc common.rs:656-672).  All values are small integers, so the
   Fq computation equals integer arithmetic; accumulate in int64. */
void or_rlc_mix(const int8_t* rho_coeffs, const int8_t* Zs, int count, int64_t m, int32_t* Zmix, int threads) {
    /* integer rot matrices */
    int32_t* rot = (int32_t*)malloc(sizeof(int32_t) * count * D * D);
    for (int i = 0; i < count; i++) {
        int32_t col[D], nxt[D];
        for (int r = 0; r < D; r++) col[r] = rho_coeffs[i * D + r];
        for (int j = 0; j < D; j++) {
            for (int r = 0; r < D; r++) rot[(size_t)i * D * D + r * D + j] = col[r];
            int32_t last = col[D - 1];
            nxt[0] = -last;
            for (int k = 1; k < D; k++) nxt[k] = col[k - 1];
            nxt[27] -= last;
            memcpy(col, nxt, sizeof col);
        }
    }
    if (count == 1) {
        /* Pi_RLC with one input is the identity (common.rs:560-564) */
        for (int64_t x = 0; x < (int64_t)D * m; x++) Zmix[x] = Zs[x];
        free(rot);
        return;
    }
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(static)
#else
    (void)threads;
#endif
    for (int64_t c = 0; c < m; c++) {
        int64_t acc[D];
        memset(acc, 0, sizeof acc);
        for (int i = 0; i < count; i++) {
            const int8_t* Zi = Zs + (size_t)i * D * m;
            const int32_t* R = rot + (size_t)i * D * D;
            for (int k = 0; k < D; k++) {
                int8_t z = Zi[(size_t)k * m + c];
                if (!z) continue;
                for (int r = 0; r < D; r++) acc[r] += (int64_t)R[r * D + k] * z;
            }
        }
        for (int r = 0; r < D; r++) Zmix[(size_t)r * m + c] = (int32_t)acc[r];
    }
    free(rot);
}

/* balanced_divrem_i64 (common.rs:44-58) */
static inline void balanced_divrem(int64_t v, int64_t b, int64_t* r_out, int64_t* q_out) {
    int64_t r = v % b;
    int64_t q = (v - r) / b;
    int64_t half = b / 2;
    if (r > half) { r -= b; q += 1; }
    else if (r < -half) { r += b; q -= 1; }
    *r_out = r; *q_out = q;
}

/* split_b_matrix_k_with_nonzero_flags (common.rs:75-268) */
int or_split_b(const int32_t* Zmix, int64_t len, int k, int b, int8_t* planes, uint8_t* nonzero) {
    int64_t B = 1;
    for (int i = 0; i < k; i++) B *= b;
    memset(planes, 0, (size_t)k * len);
    memset(nonzero, 0, (size_t)k);
    for (int64_t idx = 0; idx < len; idx++) {
        int64_t v = Zmix[idx];
        if (v >= B || v <= -B) return -1;
        for (int i = 0; i < k; i++) {
            if (v == 0) break;
            int64_t r, q;
            balanced_divrem(v, b, &r, &q);
            if (r != 0) { planes[(size_t)i * len + idx] = (int8_t)r; nonzero[i] = 1; }
            v = q;
        }
        if (v != 0) return -1;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Sum-check helpers (sumcheck.rs:48-118)                                    */
/* ------------------------------------------------------------------------ */
static kq poly_eval(const kq* c, int n, kq x) {
    if (n == 0) return K0;
    kq r = c[n - 1];
    for (int i = n - 2; i >= 0; i--) r = kadd(kmul(r, x), c[i]);
    return r;
}
void or_poly_eval_k(const uint64_t* coeffs, int n, const uint64_t* x, uint64_t* out) {
    kstore(out, poly_eval((const kq*)coeffs, n, kload(x)));
}
static void interpolate(const kq* xs, const kq* ys, int n, kq* coeffs) {
    for (int i = 0; i < n; i++) coeffs[i] = K0;
    kq numer[32], next[32];
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < n; d++) numer[d] = K0;
        numer[0] = K1;
        int cur = 0;
        for (int j = 0; j < n; j++) {
            if (i == j) continue;
            kq xj = xs[j];
            for (int d = 0; d < n; d++) next[d] = K0;
            for (int d = 0; d <= cur; d++) {
                next[d + 1] = kadd(next[d + 1], numer[d]);
                next[d] = kadd(next[d], kmul(kneg(xj), numer[d]));
            }
            memcpy(numer, next, sizeof(kq) * n);
            cur++;
        }
        kq den = K1;
        for (int j = 0; j < n; j++) if (i != j) den = kmul(den, ksub(xs[i], xs[j]));
        kq sc = kmul(ys[i], kinv(den));
        for (int d = 0; d <= cur; d++) coeffs[d] = kadd(coeffs[d], kmul(sc, numer[d]));
    }
}
void or_interpolate(const uint64_t* xs, const uint64_t* ys, int n, uint64_t* coeffs) {
    interpolate((const kq*)xs, (const kq*)ys, n, (kq*)coeffs);
}

/* chi_tail_weights (oracle.rs:1525-1540): w[mask] = prod_i (bit_i ? b_i : 1-b_i) */
static kq* chi_table(const kq* bits, int nbits) {
    size_t len = (size_t)1 << nbits;
    kq* w = (kq*)calloc(len, sizeof(kq));
    w[0] = K1;
    for (int i = 0; i < nbits; i++) {
        size_t step = (size_t)1 << i;
        kq om = ksub(K1, bits[i]);
        for (size_t mask = 0; mask < step; mask++) {
            kq v = w[mask];
            w[mask] = kmul(v, om);
            w[mask + step] = kmul(v, bits[i]);
        }
    }
    return w;
}
void or_chi_table(const uint64_t* bits, int nbits, uint64_t* out) {
    kq* w = chi_table((const kq*)bits, nbits);
    memcpy(out, w, sizeof(kq) << nbits);
    free(w);
}
static kq eq_points_bool_mask(size_t mask, const kq* pts, int n) {
    kq p = K1;
    for (int i = 0; i < n; i++) p = kmul(p, ((mask >> i) & 1) ? pts[i] : ksub(K1, pts[i]));
    return p;
}
static inline kq eq_lin(kq a, kq b) {
    return kadd(kmul(ksub(K1, a), ksub(K1, b)), kmul(a, b));
}
static kq eq_points(const kq* p, const kq* q, int n) {
    kq acc = K1;
    for (int i = 0; i < n; i++) acc = kmul(acc, eq_lin(p[i], q[i]));
    return acc;
}

/* ------------------------------------------------------------------------ */
/* CCS helpers                                                               */
/* ------------------------------------------------------------------------ */
/* out[r] += coeff * (M_j x)[r] for r < n (CSC scatter, oracle.rs:206-236) */
static void ccs_matvec_acc(const or_ccs* s, int j, const kq* x, kq coeff, kq* out) {
    uint32_t n = s->n, m = s->m;
    if (s->is_identity[j]) {
        uint32_t cap = n < m ? n : m;
        for (uint32_t r = 0; r < cap; r++) out[r] = kadd(out[r], kmul(coeff, x[r]));
        return;
    }
    const uint64_t* cp = s->col_ptr + (size_t)j * (m + 1);
    const uint32_t* ri = s->row_idx + s->nnz_off[j];
    const uint64_t* vv = s->vals + s->nnz_off[j];
    for (uint32_t c = 0; c < m; c++) {
        if (kiszero(x[c])) continue;
        kq sx = kmul(coeff, x[c]);
        for (uint64_t k = cp[c]; k < cp[c + 1]; k++) {
            uint32_t r = ri[k];
            if (r < n) out[r] = kadd(out[r], kscale(sx, vv[k]));
        }
    }
}
/* v[c] = (M_j^T chi)[c] (oracle.rs:1694-1728) */
static void ccs_matTvec(const or_ccs* s, int j, const kq* chi, size_t chi_len, kq* v) {
    uint32_t n = s->n, m = s->m;
    size_t n_eff = n < chi_len ? n : chi_len;
    for (uint32_t c = 0; c < m; c++) v[c] = K0;
    if (s->is_identity[j]) {
        size_t cap = m < n_eff ? m : n_eff;
        for (size_t c = 0; c < cap; c++) v[c] = chi[c];
        return;
    }
    const uint64_t* cp = s->col_ptr + (size_t)j * (m + 1);
    const uint32_t* ri = s->row_idx + s->nnz_off[j];
    const uint64_t* vv = s->vals + s->nnz_off[j];
    for (uint32_t c = 0; c < m; c++) {
        kq acc = K0;
        for (uint64_t k = cp[c]; k < cp[c + 1]; k++) {
            uint32_t r = ri[k];
            if (r < n_eff) acc = kadd(acc, kscale(chi[r], vv[k]));
        }
        v[c] = acc;
    }
}
/* f.eval_in_ext */
static kq f_eval(const or_ccs* s, const kq* mv) {
    kq acc = K0;
    for (uint32_t tt = 0; tt < s->n_terms; tt++) {
        kq p = kfq(s->f_coeff[tt]);
        for (uint32_t j = 0; j < s->t; j++) {
            uint32_t e = s->f_exps[(size_t)tt * s->t + j];
            for (uint32_t q = 0; q < e; q++) p = kmul(p, mv[j]);
        }
        acc = kadd(acc, p);
    }
    return acc;
}
static inline kq range_product_b2(kq y) { return kmul(y, ksub(kmul(y, y), K1)); }

/* ------------------------------------------------------------------------ */
/* Pi_CCS optimized oracle (oracle.rs)                                       */
/* ------------------------------------------------------------------------ */
struct or_ccs_oracle {
    const or_ccs* s;   /* caller keeps alive */
    int k, b, ell_d, ell_n, d_sc;
    int64_t m;
    const int8_t* Z;   /* caller keeps alive: [k][54][m] */
    kq *alpha, *beta_a, *beta_r, gamma, *r_inputs;
    int has_inputs;
    /* row stream */
    size_t cur_len;
    kq *eq_beta_r, *eq_rin, *z1, **fvar, *nc, *wg, *eval_tbl, gamma_to_k;
    int n_fvar, *fvar_j;
    int deg_max;
    /* rounds */
    int round_idx;
    kq *row_chals, *ajtai_chals;
    /* ajtai precomp */
    int have_pre;
    kq *y_nc;   /* [k][D] */
    kq *y_eval; /* [k][t][D] */
    kq f_prime, pre_eq_beta_r, pre_eq_rin;
};

static kq* kdup(const uint64_t* src, int n) {
    kq* d = (kq*)malloc(sizeof(kq) * (n > 0 ? n : 1));
    for (int i = 0; i < n; i++) d[i] = kload(src + 2 * i);
    return d;
}

or_ccs_oracle* or_ccs_oracle_new(const or_ccs* s, const int8_t* Z, int k, int b,
                                 const uint64_t* alpha, const uint64_t* beta_a, const uint64_t* beta_r,
                                 const uint64_t* gamma, const uint64_t* r_inputs,
                                 int ell_d, int ell_n, int d_sc) {
    if (b != 2 || k < 1) return NULL;
    or_ccs_oracle* o = (or_ccs_oracle*)calloc(1, sizeof(*o));
    o->s = s; o->k = k; o->b = b; o->ell_d = ell_d; o->ell_n = ell_n; o->d_sc = d_sc;
    o->m = s->m; o->Z = Z;
    o->alpha = kdup(alpha, ell_d); o->beta_a = kdup(beta_a, ell_d); o->beta_r = kdup(beta_r, ell_n);
    o->gamma = kload(gamma);
    o->has_inputs = r_inputs != NULL;
    o->r_inputs = r_inputs ? kdup(r_inputs, ell_n) : NULL;
    o->row_chals = (kq*)calloc(ell_n + 1, sizeof(kq));
    o->ajtai_chals = (kq*)calloc(ell_d + 1, sizeof(kq));
    size_t n_pad = (size_t)1 << ell_n;
    size_t n_eff = s->n;
    size_t m = s->m;
    o->cur_len = n_pad;
    o->eq_beta_r = chi_table(o->beta_r, ell_n);
    o->eq_rin = o->has_inputs ? chi_table(o->r_inputs, ell_n) : NULL;

    /* compile f: used variables (oracle.rs:136-186) */
    int t = s->t;
    o->fvar_j = (int*)calloc(t, sizeof(int));
    int fmaxdeg = 0;
    for (int j = 0; j < t; j++) {
        int used = 0;
        for (uint32_t tt = 0; tt < s->n_terms; tt++) if (s->f_exps[tt * t + j]) used = 1;
        if (used) o->fvar_j[o->n_fvar++] = j;
    }
    for (uint32_t tt = 0; tt < s->n_terms; tt++) {
        int dg = 0;
        for (int j = 0; j < t; j++) dg += s->f_exps[tt * t + j];
        if (dg > fmaxdeg) fmaxdeg = dg;
    }
    o->deg_max = fmaxdeg + 1 > 4 ? fmaxdeg + 1 : 4;

    /* w_gamma_nc[i*D+rho] = chi_{beta_a}[rho] * gamma^(i+1)  (oracle.rs:196-213) */
    o->wg = (kq*)calloc((size_t)k * D, sizeof(kq));
    {
        kq g = o->gamma;
        for (int i = 0; i < k; i++) {
            for (int rho = 0; rho < D; rho++)
                o->wg[i * D + rho] = kmul(eq_points_bool_mask(rho, o->beta_a, ell_d), g);
            g = kmul(g, o->gamma);
        }
    }
    /* z1 (oracle.rs:215-243) */
    o->z1 = (kq*)calloc(m, sizeof(kq));
    {
        uint64_t pw[D]; pw[0] = 1;
        for (int r = 1; r < D; r++) pw[r] = fq_mul(pw[r - 1], (uint64_t)b);
        for (int rho = 0; rho < D; rho++)
            for (size_t c = 0; c < m; c++)
                o->z1[c] = kadd(o->z1[c], kfq(fq_mul(fq_from_i64(Z[rho * m + c]), pw[rho])));
    }
    /* f-var tables (oracle.rs:245-285) */
    o->fvar = (kq**)calloc(o->n_fvar > 0 ? o->n_fvar : 1, sizeof(kq*));
    for (int v = 0; v < o->n_fvar; v++) {
        o->fvar[v] = (kq*)calloc(n_pad, sizeof(kq));
        ccs_matvec_acc(s, o->fvar_j[v], o->z1, K1, o->fvar[v]);
    }
    /* NC tables: nc[(i*n_pad + row)*D + rho] (oracle.rs:287-308) */
    o->nc = (kq*)calloc((size_t)k * n_pad * D, sizeof(kq));
    {
        size_t cap = n_eff < n_pad ? n_eff : n_pad;
        if (cap > m) cap = m;
        for (int i = 0; i < k; i++)
            for (size_t row = 0; row < cap; row++)
                for (int rho = 0; rho < D; rho++)
                    o->nc[((size_t)i * n_pad + row) * D + rho] = kfq(fq_from_i64(Z[((size_t)i * D + rho) * m + row]));
    }
    /* gamma^k and Eval table (oracle.rs:310-393) */
    o->gamma_to_k = K1;
    for (int i = 0; i < k; i++) o->gamma_to_k = kmul(o->gamma_to_k, o->gamma);
    if (k >= 2 && o->has_inputs) {
        kq w_alpha[D];
        for (int rho = 0; rho < D; rho++) w_alpha[rho] = eq_points_bool_mask(rho, o->alpha, ell_d);
        o->eval_tbl = (kq*)calloc(n_pad, sizeof(kq));
        kq* s_alpha = (kq*)calloc(m, sizeof(kq));
        kq gpi = K1;
        for (int i = 1; i < k; i++) {
            gpi = kmul(gpi, o->gamma);
            for (size_t c = 0; c < m; c++) s_alpha[c] = K0;
            for (int rho = 0; rho < D; rho++) {
                for (size_t c = 0; c < m; c++) {
                    int8_t z = Z[((size_t)i * D + rho) * m + c];
                    if (z) s_alpha[c] = kadd(s_alpha[c], kscale(w_alpha[rho], fq_from_i64(z)));
                }
            }
            kq gkj = K1;
            for (int j = 0; j < t; j++) {
                kq coeff = kmul(gpi, gkj);
                ccs_matvec_acc(s, j, s_alpha, coeff, o->eval_tbl);
                gkj = kmul(gkj, o->gamma_to_k);
            }
        }
        free(s_alpha);
    }
    return o;
}

void or_ccs_oracle_free(or_ccs_oracle* o) {
    if (!o) return;
    free(o->alpha); free(o->beta_a); free(o->beta_r); free(o->r_inputs);
    free(o->row_chals); free(o->ajtai_chals);
    free(o->eq_beta_r); free(o->eq_rin); free(o->z1);
    for (int v = 0; v < o->n_fvar; v++) free(o->fvar[v]);
    free(o->fvar); free(o->fvar_j); free(o->nc); free(o->wg); free(o->eval_tbl);
    free(o->y_nc); free(o->y_eval);
    free(o);
}
int or_ccs_oracle_num_rounds(const or_ccs_oracle* o) { return o->ell_n + o->ell_d; }

/* poly_mul_affine_inplace (oracle.rs:1036-1045) */
static void poly_mul_affine(kq* poly, int len, kq a, kq b) {
    kq prev = K0;
    for (int i = 0; i < len; i++) {
        kq old = poly[i];
        poly[i] = kadd(kmul(a, old), kmul(b, prev));
        prev = old;
    }
}

/* evals_row_phase_impl, b=2 generic K path (oracle.rs:1047-1178); the pair
   loop is split across threads like the reference's rayon fold/reduce
   (oracle.rs:542-658), exact arithmetic makes the split invisible. */
static void row_pair_accum(or_ccs_oracle* o, size_t t, kq* coeffs) {
    const or_ccs* s = o->s;
    size_t L = o->cur_len;
    int dm = o->deg_max;
    kq inner[16], tp[16];
    kq three = kfq(3);
    kq e0 = o->eq_beta_r[2 * t];
    kq e1 = ksub(o->eq_beta_r[2 * t + 1], e0);
    for (int i = 0; i <= dm; i++) inner[i] = K0;
    for (uint32_t tt = 0; tt < s->n_terms; tt++) {
        for (int i = 0; i <= dm; i++) tp[i] = K0;
        tp[0] = kfq(s->f_coeff[tt]);
        for (int v = 0; v < o->n_fvar; v++) {
            uint32_t e = s->f_exps[tt * s->t + o->fvar_j[v]];
            if (!e) continue;
            kq a = o->fvar[v][2 * t];
            kq bb = ksub(o->fvar[v][2 * t + 1], a);
            for (uint32_t q = 0; q < e; q++) poly_mul_affine(tp, dm + 1, a, bb);
        }
        for (int i = 0; i <= dm; i++) inner[i] = kadd(inner[i], tp[i]);
    }
    for (int w = 0; w < o->k; w++) {
        const kq* lo = o->nc + ((size_t)w * L + 2 * t) * D;
        const kq* hi = lo + D;
        for (int rho = 0; rho < D; rho++) {
            kq wg = o->wg[w * D + rho];
            kq a = lo[rho];
            kq bb = ksub(hi[rho], a);
            kq a2 = kmul(a, a), a3 = kmul(a2, a), b2 = kmul(bb, bb), b3 = kmul(b2, bb);
            kq t0 = ksub(a3, a);
            kq t1 = ksub(kmul(kmul(a2, bb), three), bb);
            kq t2 = kmul(kmul(a, b2), three);
            kq t3 = b3;
            inner[0] = kadd(inner[0], kmul(wg, t0));
            inner[1] = kadd(inner[1], kmul(wg, t1));
            inner[2] = kadd(inner[2], kmul(wg, t2));
            inner[3] = kadd(inner[3], kmul(wg, t3));
        }
    }
    coeffs[0] = kadd(coeffs[0], kmul(e0, inner[0]));
    for (int d = 1; d <= dm; d++)
        coeffs[d] = kadd(coeffs[d], kadd(kmul(e0, inner[d]), kmul(e1, inner[d - 1])));
    if (o->eq_rin && o->eval_tbl) {
        kq r0 = o->eq_rin[2 * t], r1 = ksub(o->eq_rin[2 * t + 1], r0);
        kq v0 = o->eval_tbl[2 * t], v1 = ksub(o->eval_tbl[2 * t + 1], v0);
        kq g = o->gamma_to_k;
        coeffs[0] = kadd(coeffs[0], kmul(g, kmul(r0, v0)));
        coeffs[1] = kadd(coeffs[1], kmul(g, kadd(kmul(r0, v1), kmul(r1, v0))));
        coeffs[2] = kadd(coeffs[2], kmul(g, kmul(r1, v1)));
    }
}

static void evals_row_phase(or_ccs_oracle* o, const kq* xs, int nx, kq* ys) {
    size_t tail = o->cur_len / 2;
    int dm = o->deg_max;
    kq coeffs[16];
    for (int i = 0; i <= dm; i++) coeffs[i] = K0;
#ifdef _OPENMP
#pragma omp parallel if (tail >= 1024)
#endif
    {
        kq local[16];
        for (int i = 0; i <= dm; i++) local[i] = K0;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (size_t t = 0; t < tail; t++) row_pair_accum(o, t, local);
#ifdef _OPENMP
#pragma omp critical
#endif
        for (int i = 0; i <= dm; i++) coeffs[i] = kadd(coeffs[i], local[i]);
    }
    for (int i = 0; i < nx; i++) ys[i] = poly_eval(coeffs, dm + 1, xs[i]);
}

static void fold_tbl(kq* T, size_t len, kq r) {
    size_t half = len / 2;
    for (size_t i = 0; i < half; i++) T[i] = kadd(T[2 * i], kmul(ksub(T[2 * i + 1], T[2 * i]), r));
}

/* RowStreamState::fold_inplace (oracle.rs:470-503) */
static void row_fold(or_ccs_oracle* o, kq r) {
    size_t L = o->cur_len, half = L / 2;
    fold_tbl(o->eq_beta_r, L, r);
    if (o->eq_rin) fold_tbl(o->eq_rin, L, r);
    for (int v = 0; v < o->n_fvar; v++) fold_tbl(o->fvar[v], L, r);
    for (int w = 0; w < o->k; w++) {
        kq* base = o->nc + (size_t)w * L * D;          /* old layout stride L */
        kq* dst = o->nc + (size_t)w * half * D;        /* compact to stride half */
        /* w == 0 folds in place front to back: element i reads 2i, 2i+1 >= i,
           so only a serial loop is safe there; w >= 1 writes below its source */
#ifdef _OPENMP
#pragma omp parallel for schedule(static) if (w > 0 && half >= 4096)
#endif
        for (size_t i = 0; i < half; i++)
            for (int rho = 0; rho < D; rho++) {
                kq lo = base[(2 * i) * D + rho], hi = base[(2 * i + 1) * D + rho];
                dst[i * D + rho] = kadd(lo, kmul(ksub(hi, lo), r));
            }
    }
    if (o->eval_tbl) fold_tbl(o->eval_tbl, L, r);
    o->cur_len = half;
}

/* precompute_for_r (oracle.rs:1659-1783) */
static void precompute_for_r(or_ccs_oracle* o) {
    const or_ccs* s = o->s;
    int t = s->t, k = o->k;
    size_t m = s->m;
    kq* chi_r = chi_table(o->row_chals, o->ell_n);
    size_t n_sz = (size_t)1 << o->ell_n;
    o->pre_eq_beta_r = eq_points(o->row_chals, o->beta_r, o->ell_n);
    o->pre_eq_rin = o->has_inputs ? eq_points(o->row_chals, o->r_inputs, o->ell_n) : K0;
    kq* vj = (kq*)calloc((size_t)t * m, sizeof(kq));
    for (int j = 0; j < t; j++) ccs_matTvec(s, j, chi_r, n_sz, vj + (size_t)j * m);
    kq mv[64];
    for (int j = 0; j < t; j++) {
        kq acc = K0;
        for (size_t c = 0; c < m; c++) acc = kadd(acc, kmul(o->z1[c], vj[(size_t)j * m + c]));
        mv[j] = acc;
    }
    o->f_prime = f_eval(s, mv);
    o->y_nc = (kq*)calloc((size_t)k * D, sizeof(kq));
    o->y_eval = (kq*)calloc((size_t)k * t * D, sizeof(kq));
#ifdef _OPENMP
#pragma omp parallel for collapse(3) schedule(dynamic)
#endif
    for (int i = 0; i < k; i++) {
        for (int j = 0; j < t; j++) {
            for (int rho = 0; rho < D; rho++) {
                const int8_t* zr = o->Z + ((size_t)i * D + rho) * m;
                kq acc = K0;
                for (size_t c = 0; c < m; c++) {
                    if (zr[c] == 1) acc = kadd(acc, vj[(size_t)j * m + c]);
                    else if (zr[c] == -1) acc = ksub(acc, vj[(size_t)j * m + c]);
                    else if (zr[c]) acc = kadd(acc, kscale(vj[(size_t)j * m + c], fq_from_i64(zr[c])));
                }
                o->y_eval[((size_t)i * t + j) * D + rho] = acc;
            }
        }
    }
    /* NC uses v_1 = chi_r restricted (matrix 0 is the identity) */
    for (int i = 0; i < k; i++) memcpy(o->y_nc + (size_t)i * D, o->y_eval + ((size_t)i * t + 0) * D, sizeof(kq) * D);
    free(vj); free(chi_r);
    o->have_pre = 1;
}

/* fold_bit_inplace (oracle.rs:1447-1468) */
static void fold_bit_inplace(kq* dg, int bit, kq a) {
    int stride = 1 << bit, step = stride << 1;
    for (int base = 0; base < D; base += step)
        for (int off = 0; off < stride; off++) {
            int i0 = base + off;
            if (i0 >= D) break;
            int i1 = i0 + stride;
            kq lo = dg[i0], hi = i1 < D ? dg[i1] : K0;
            dg[i0] = kadd(lo, kmul(ksub(hi, lo), a));
        }
}

/* evals_ajtai_phase (oracle.rs:1812-1951) */
static void evals_ajtai_phase(or_ccs_oracle* o, const kq* xs, int nx, kq* ys) {
    const or_ccs* s = o->s;
    int j = o->round_idx - o->ell_n;
    int k = o->k, t = s->t;
    if (!o->have_pre) precompute_for_r(o);
    int ntail = o->ell_d - j - 1;
    kq* wb = chi_table(o->beta_a + j + 1, ntail);
    kq* wa = chi_table(o->alpha + j + 1, ntail);
    int tail_len = 1 << ntail;
    int hs = 1 << (j + 1);
    kq ebp = K1, eap = K1;
    for (int i = 0; i < j; i++) {
        ebp = kmul(ebp, eq_lin(o->ajtai_chals[i], o->beta_a[i]));
        eap = kmul(eap, eq_lin(o->ajtai_chals[i], o->alpha[i]));
    }
    kq* gpi = (kq*)malloc(sizeof(kq) * k);
    gpi[0] = K1;
    for (int i = 1; i < k; i++) gpi[i] = kmul(gpi[i - 1], o->gamma);
    kq gk = o->gamma_to_k;
    kq gkj[64]; gkj[0] = K1;
    for (int jj = 1; jj < t; jj++) gkj[jj] = kmul(gkj[jj - 1], gk);
    kq* ync = (kq*)malloc(sizeof(kq) * k * D);
    memcpy(ync, o->y_nc, sizeof(kq) * k * D);
    for (int i = 0; i < k; i++) for (int bb = 0; bb < j; bb++) fold_bit_inplace(ync + i * D, bb, o->ajtai_chals[bb]);
    kq* yev = (kq*)malloc(sizeof(kq) * k * t * D);
    memcpy(yev, o->y_eval, sizeof(kq) * k * t * D);
    for (int q = 0; q < k * t; q++) for (int bb = 0; bb < j; bb++) fold_bit_inplace(yev + q * D, bb, o->ajtai_chals[bb]);
    kq beta_j = o->beta_a[j], alpha_j = o->alpha[j];
    for (int xi = 0; xi < nx; xi++) {
        kq x = xs[xi];
        kq eq_beta = kmul(o->pre_eq_beta_r, kmul(ebp, eq_lin(x, beta_j)));
        kq eq_ar = o->has_inputs ? kmul(o->pre_eq_rin, kmul(eap, eq_lin(x, alpha_j))) : K0;
        kq nc_sum = K0, g = o->gamma;
        kq tmp[D];
        for (int i = 0; i < k; i++) {
            memcpy(tmp, ync + i * D, sizeof tmp);
            fold_bit_inplace(tmp, j, x);
            kq acc = K0;
            for (int tt = 0; tt < tail_len; tt++) {
                int idx = tt * hs;
                if (idx < D) acc = kadd(acc, kmul(wb[tt], range_product_b2(tmp[idx])));
            }
            nc_sum = kadd(nc_sum, kmul(g, acc));
            g = kmul(g, o->gamma);
        }
        kq out = kmul(eq_beta, kadd(o->f_prime, nc_sum));
        if (k >= 2 && !kiszero(eq_ar)) {
            kq inner = K0;
            for (int jm = 0; jm < t; jm++) {
                kq sum_j = K0;
                for (int i = 1; i < k; i++) {
                    memcpy(tmp, yev + (i * t + jm) * D, sizeof tmp);
                    fold_bit_inplace(tmp, j, x);
                    kq ydot = K0;
                    for (int tt = 0; tt < tail_len; tt++) {
                        int idx = tt * hs;
                        if (idx < D) ydot = kadd(ydot, kmul(wa[tt], tmp[idx]));
                    }
                    sum_j = kadd(sum_j, kmul(kmul(gpi[i], gkj[jm]), ydot));
                }
                inner = kadd(inner, sum_j);
            }
            out = kadd(out, kmul(eq_ar, kmul(gk, inner)));
        }
        ys[xi] = out;
    }
    free(wb); free(wa); free(gpi); free(ync); free(yev);
}

void or_ccs_oracle_evals(or_ccs_oracle* o, const uint64_t* xs, int nx, uint64_t* ys) {
    if (o->round_idx < o->ell_n) evals_row_phase(o, (const kq*)xs, nx, (kq*)ys);
    else evals_ajtai_phase(o, (const kq*)xs, nx, (kq*)ys);
}
void or_ccs_oracle_fold(or_ccs_oracle* o, const uint64_t* r) {
    kq rr = kload(r);
    if (o->round_idx < o->ell_n) {
        o->row_chals[o->round_idx] = rr;
        row_fold(o, rr);
    } else {
        o->ajtai_chals[o->round_idx - o->ell_n] = rr;
    }
    o->round_idx++;
}
/* build_me_outputs_from_ajtai_precomp (oracle.rs:1955-2072): y digits + y_scalars */
void or_ccs_oracle_me_outputs(or_ccs_oracle* o, uint64_t* y_out, uint64_t* y_scalars) {
    if (!o->have_pre) precompute_for_r(o);
    int t = o->s->t;
    uint64_t pw[D]; pw[0] = 1;
    for (int r = 1; r < D; r++) pw[r] = fq_mul(pw[r - 1], (uint64_t)o->b);
    for (int i = 0; i < o->k; i++)
        for (int j = 0; j < t; j++) {
            const kq* dg = o->y_eval + ((size_t)i * t + j) * D;
            kq acc = K0;
            for (int rho = 0; rho < D; rho++) {
                kstore(y_out + 2 * (((size_t)i * t + j) * D + rho), dg[rho]);
                acc = kadd(acc, kscale(dg[rho], pw[rho]));
            }
            kstore(y_scalars + 2 * ((size_t)i * t + j), acc);
        }
}

/* run_sumcheck_prover with externally fixed challenges (sumcheck.rs:124-209) */
int or_ccs_sumcheck_fixed(or_ccs_oracle* o, const uint64_t* initial_sum, const uint64_t* chals,
                          uint64_t* evals_out, uint64_t* final_sum) {
    int rounds = or_ccs_oracle_num_rounds(o);
    int np = o->d_sc + 1;
    kq xs[32], ys[32], co[32];
    for (int i = 0; i < np; i++) xs[i] = kfq((uint64_t)i);
    kq running = kload(initial_sum);
    for (int r = 0; r < rounds; r++) {
        or_ccs_oracle_evals(o, (const uint64_t*)xs, np, (uint64_t*)ys);
        if (evals_out) memcpy(evals_out + (size_t)r * np * 2, ys, sizeof(kq) * np);
        if (!keq(kadd(ys[0], ys[1]), running)) return -1 - r;
        interpolate(xs, ys, np, co);
        kq c = kload(chals + 2 * r);
        running = poly_eval(co, np, c);
        or_ccs_oracle_fold(o, chals + 2 * r);
    }
    kstore(final_sum, running);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Paper-exact Q (paper_exact.rs:136-340, 414-687)                           */
/* ------------------------------------------------------------------------ */
static kq csc_get(const or_ccs* s, int j, uint32_t row, uint32_t col) {
    if (s->is_identity[j]) return (row == col && row < s->n) ? K1 : K0;
    const uint64_t* cp = s->col_ptr + (size_t)j * (s->m + 1);
    const uint32_t* ri = s->row_idx + s->nnz_off[j];
    const uint64_t* vv = s->vals + s->nnz_off[j];
    uint64_t acc = 0;
    for (uint64_t k = cp[col]; k < cp[col + 1]; k++) if (ri[k] == row) acc = fq_add(acc, vv[k]);
    return kfq(acc);
}

void or_q_sum_hypercube(const or_ccs* s, const int8_t* Z, int k, int b,
                        const uint64_t* alpha_, const uint64_t* beta_a_, const uint64_t* beta_r_,
                        const uint64_t* gamma_, const uint64_t* r_inputs_, int ell_d, int ell_n, uint64_t* out) {
    (void)b;
    const kq* alpha = (const kq*)alpha_; const kq* beta_a = (const kq*)beta_a_;
    const kq* beta_r = (const kq*)beta_r_; kq gamma = kload(gamma_);
    const kq* rin = (const kq*)r_inputs_;
    size_t m = s->m;
    int t = s->t;
    uint64_t* z1 = (uint64_t*)malloc(8 * m);
    or_recompose_b2(Z, m, z1);
    kq gk = K1;
    for (int i = 0; i < k; i++) gk = kmul(gk, gamma);
    kq total = K0;
    for (size_t xr = 0; xr < ((size_t)1 << ell_n); xr++) {
        /* F(xr) */
        kq mv[64];
        for (int j = 0; j < t; j++) {
            kq acc = K0;
            if (xr < s->n)
                for (size_t c = 0; c < m; c++) acc = kadd(acc, kmul(csc_get(s, j, xr, c), kfq(z1[c])));
            mv[j] = acc;
        }
        kq Fv = f_eval(s, mv);
        kq eqr = eq_points_bool_mask(xr, beta_r, ell_n);
        kq eqrin = rin ? eq_points_bool_mask(xr, rin, ell_n) : K0;
        for (size_t xa = 0; xa < ((size_t)1 << ell_d); xa++) {
            kq eq_beta = kmul(eq_points_bool_mask(xa, beta_a, ell_d), eqr);
            kq nc = K0, g = gamma;
            for (int i = 0; i < k; i++) {
                kq y = K0;
                if (xa < D && xr < m && xr < s->n) y = kfq(fq_from_i64(Z[((size_t)i * D + xa) * m + xr]));
                nc = kadd(nc, kmul(g, range_product_b2(y)));
                g = kmul(g, gamma);
            }
            kq acc = kmul(eq_beta, kadd(Fv, nc));
            if (rin && k >= 2) {
                kq eq_ar = kmul(eq_points_bool_mask(xa, alpha, ell_d), eqrin);
                kq inner = K0;
                kq gkj = K1;
                for (int j = 0; j < t; j++) {
                    kq w = gkj;
                    for (int i = 1; i < k; i++) {
                        w = kmul(w, gamma); /* gamma^i * gk^j */
                        kq y = K0;
                        if (xa < D && xr < s->n)
                            for (size_t c = 0; c < m; c++) {
                                int8_t z = Z[((size_t)i * D + xa) * m + c];
                                if (z) y = kadd(y, kscale(csc_get(s, j, xr, c), fq_from_i64(z)));
                            }
                        inner = kadd(inner, kmul(w, kmul(eq_ar, y)));
                    }
                    gkj = kmul(gkj, gk);
                }
                acc = kadd(acc, kmul(gk, inner));
            }
            total = kadd(total, acc);
        }
    }
    free(z1);
    kstore(out, total);
}

void or_q_eval_ext(const or_ccs* s, const int8_t* Z, int k, int b,
                   const uint64_t* alpha_, const uint64_t* beta_a_, const uint64_t* beta_r_,
                   const uint64_t* gamma_, const uint64_t* r_inputs_, int ell_d, int ell_n,
                   const uint64_t* alpha_p_, const uint64_t* r_p_, uint64_t* out) {
    (void)b;
    const kq* alpha = (const kq*)alpha_; const kq* beta_a = (const kq*)beta_a_;
    const kq* beta_r = (const kq*)beta_r_; kq gamma = kload(gamma_);
    const kq* rin = (const kq*)r_inputs_;
    const kq* ap = (const kq*)alpha_p_; const kq* rp = (const kq*)r_p_;
    size_t m = s->m;
    int t = s->t;
    size_t n_sz = (size_t)1 << ell_n;
    kq* chi_a = chi_table(ap, ell_d);
    kq* chi_r = chi_table(rp, ell_n);
    kq eq_beta = kmul(eq_points(ap, beta_a, ell_d), eq_points(rp, beta_r, ell_n));
    kq eq_ar = rin ? kmul(eq_points(ap, alpha, ell_d), eq_points(rp, rin, ell_n)) : K0;
    uint64_t* z1 = (uint64_t*)malloc(8 * m);
    or_recompose_b2(Z, m, z1);
    kq* zk = (kq*)malloc(sizeof(kq) * m);
    for (size_t c = 0; c < m; c++) zk[c] = kfq(z1[c]);
    kq* vj = (kq*)malloc(sizeof(kq) * m);
    kq mv[64];
    for (int j = 0; j < t; j++) {
        ccs_matTvec(s, j, chi_r, n_sz, vj);
        kq acc = K0;
        for (size_t c = 0; c < m; c++) acc = kadd(acc, kmul(vj[c], zk[c]));
        mv[j] = acc;
    }
    kq Fp = f_eval(s, mv);
    kq gk = K1;
    for (int i = 0; i < k; i++) gk = kmul(gk, gamma);
    /* NC with v1 = M_0^T chi_r */
    ccs_matTvec(s, 0, chi_r, n_sz, vj);
    kq nc = K0, g = gamma;
    for (int i = 0; i < k; i++) {
        kq ye = K0;
        for (int rho = 0; rho < D && rho < (1 << ell_d); rho++) {
            kq acc = K0;
            const int8_t* zr = Z + ((size_t)i * D + rho) * m;
            for (size_t c = 0; c < m; c++) if (zr[c]) acc = kadd(acc, kscale(vj[c], fq_from_i64(zr[c])));
            ye = kadd(ye, kmul(acc, chi_a[rho]));
        }
        nc = kadd(nc, kmul(g, range_product_b2(ye)));
        g = kmul(g, gamma);
    }
    kq ev = K0;
    if (k >= 2) {
        for (int j = 0; j < t; j++) {
            ccs_matTvec(s, j, chi_r, n_sz, vj);
            for (int i = 1; i < k; i++) {
                kq ye = K0;
                for (int rho = 0; rho < D && rho < (1 << ell_d); rho++) {
                    kq acc = K0;
                    const int8_t* zr = Z + ((size_t)i * D + rho) * m;
                    for (size_t c = 0; c < m; c++) if (zr[c]) acc = kadd(acc, kscale(vj[c], fq_from_i64(zr[c])));
                    ye = kadd(ye, kmul(acc, chi_a[rho]));
                }
                kq w = K1;
                for (int q = 0; q < i; q++) w = kmul(w, gamma);
                for (int q = 0; q < j; q++) w = kmul(w, gk);
                ev = kadd(ev, kmul(w, ye));
            }
        }
    }
    kq lhs = kadd(kmul(eq_beta, kadd(Fp, nc)), kmul(eq_ar, kmul(gk, ev)));
    kstore(out, lhs);
    free(chi_a); free(chi_r); free(z1); free(zk); free(vj);
}

/* compute_y_from_Z_and_r (common.rs:582-650): y_j = Z (M_j^T chi_r) */
void or_me_y_at_r(const or_ccs* s, const int8_t* Z, int ell_n, const uint64_t* r, int b,
                  uint64_t* y, uint64_t* y_scalars) {
    size_t m = s->m;
    int t = s->t;
    kq* chi = chi_table((const kq*)r, ell_n);
    kq* vj = (kq*)malloc(sizeof(kq) * m);
    uint64_t pw[D]; pw[0] = 1;
    for (int q = 1; q < D; q++) pw[q] = fq_mul(pw[q - 1], (uint64_t)b);
    for (int j = 0; j < t; j++) {
        ccs_matTvec(s, j, chi, (size_t)1 << ell_n, vj);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) if (m >= 4096)
#endif
        for (int rho = 0; rho < D; rho++) {
            kq acc = K0;
            const int8_t* zr = Z + (size_t)rho * m;
            for (size_t c = 0; c < m; c++) if (zr[c]) acc = kadd(acc, kscale(vj[c], fq_from_i64(zr[c])));
            kstore(y + 2 * ((size_t)j * D + rho), acc);
        }
        kq sc = K0;
        for (int rho = 0; rho < D; rho++) sc = kadd(sc, kscale(kload(y + 2 * ((size_t)j * D + rho)), pw[rho]));
        kstore(y_scalars + 2 * j, sc);
    }
    free(chi); free(vj);
}

/* ------------------------------------------------------------------------ */
/* Transcript: Poseidon2 width-8 overwrite sponge                            */
/* (crates/neo-transcript/src/poseidon2.rs:10-310).  Permutation restated     */
/* from the Poseidon2 paper (eprint 2023/323): t=8, x^7, R_F=8, R_P=22,       */
/* external circ(2M4, M4), internal 1 + diag(mu); constants from ChaCha8      */
/* (RFC 7539 block function, 8 rounds) seeded with the reference SEED, by     */
/* rejection sampling.  Parity unpinned (p3-poseidon2 0.4.1 not vendored).    */
/* ------------------------------------------------------------------------ */
typedef struct { uint32_t key[8]; uint64_t ctr; uint32_t blk[16]; int idx; } or_chacha;
static uint32_t rl(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }
static void cc_refill(or_chacha* c) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
    for (int i = 0; i < 8; i++) s[4 + i] = c->key[i];
    s[12] = (uint32_t)c->ctr; s[13] = (uint32_t)(c->ctr >> 32); s[14] = 0; s[15] = 0;
    uint32_t x[16];
    memcpy(x, s, sizeof x);
    static const int QI[8][4] = {{0,4,8,12},{1,5,9,13},{2,6,10,14},{3,7,11,15},{0,5,10,15},{1,6,11,12},{2,7,8,13},{3,4,9,14}};
    for (int r = 0; r < 4; r++)
        for (int q = 0; q < 8; q++) {
            uint32_t *a = &x[QI[q][0]], *b = &x[QI[q][1]], *cc = &x[QI[q][2]], *d = &x[QI[q][3]];
            *a += *b; *d ^= *a; *d = rl(*d, 16);
            *cc += *d; *b ^= *cc; *b = rl(*b, 12);
            *a += *b; *d ^= *a; *d = rl(*d, 8);
            *cc += *d; *b ^= *cc; *b = rl(*b, 7);
        }
    for (int i = 0; i < 16; i++) c->blk[i] = x[i] + s[i];
    c->ctr++;
    c->idx = 0;
}
static uint64_t cc_u64(or_chacha* c) {
    if (c->idx >= 16) cc_refill(c);
    uint64_t lo = c->blk[c->idx++];
    if (c->idx >= 16) cc_refill(c);
    uint64_t hi = c->blk[c->idx++];
    return lo | (hi << 32);
}

/* rand_core fill_bytes over a u32 block stream: whole words, little endian
   (a partial last word is consumed). */
static void cc_fill(or_chacha* c, uint8_t* out, size_t n) {
    size_t i = 0;
    while (i < n) {
        if (c->idx >= 16) cc_refill(c);
        uint32_t w = c->blk[c->idx++];
        for (int b = 0; b < 4 && i < n; b++, i++) out[i] = (uint8_t)(w >> (8 * b));
    }
}
static void cc_init(or_chacha* c, const uint8_t* seed) {
    for (int i = 0; i < 8; i++)
        c->key[i] = (uint32_t)seed[4*i] | ((uint32_t)seed[4*i+1] << 8) | ((uint32_t)seed[4*i+2] << 16) |
                    ((uint32_t)seed[4*i+3] << 24);
    c->ctr = 0; c->idx = 16;
}

/* sample_uniform_fq generalised to any bound (commit.rs:21-30): per stream the
   first counts[s] next_u64() values < bound, concatenated into out. */
void or_chacha8_sample(const uint8_t* seeds, uint32_t n_streams, const uint64_t* counts, uint64_t bound,
                       uint64_t* out) {
    uint64_t* offs = (uint64_t*)malloc(sizeof(uint64_t) * (n_streams + 1));
    offs[0] = 0;
    for (uint32_t s = 0; s < n_streams; s++) offs[s + 1] = offs[s] + counts[s];
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t s = 0; s < (int64_t)n_streams; s++) {
        or_chacha c;
        cc_init(&c, seeds + 32 * s);
        uint64_t* o = out + offs[s];
        for (uint64_t i = 0; i < counts[s]; i++) {
            uint64_t x;
            do { x = cc_u64(&c); } while (x >= bound);
            o[i] = x;
        }
    }
    free(offs);
}

/* Ajtai setup (commit.rs:133-157, mode 0) and setup_par (commit.rs:159-225,
   mode 1) with rng = ChaCha8Rng::from_seed(seed): out[(i*m + j)*54 + s]. */
void or_pp_setup(const uint8_t* seed, uint32_t kappa, uint64_t m, int mode, uint64_t* out) {
    if (mode == 0) {
        uint64_t n = (uint64_t)kappa * m * 54;
        or_chacha8_sample(seed, 1, &n, Q, out);
        return;
    }
    uint64_t chunk = m < (1u << 15) ? m : (1u << 15);
    if (chunk < 1024) chunk = 1024;
    uint64_t n_chunks = (m + chunk - 1) / chunk;
    uint8_t* seeds = (uint8_t*)malloc(32 * (size_t)kappa * n_chunks);
    uint64_t* counts = (uint64_t*)malloc(8 * (size_t)kappa * n_chunks);
    uint8_t* rows = (uint8_t*)malloc(32 * (size_t)kappa);
    or_chacha master;
    cc_init(&master, seed);
    for (uint32_t i = 0; i < kappa; i++) cc_fill(&master, rows + 32 * i, 32);
    for (uint32_t i = 0; i < kappa; i++) {
        or_chacha rr;
        cc_init(&rr, rows + 32 * i);
        for (uint64_t c = 0; c < n_chunks; c++) {
            cc_fill(&rr, seeds + 32 * (i * n_chunks + c), 32);
            uint64_t lo = c * chunk, hi = lo + chunk < m ? lo + chunk : m;
            counts[i * n_chunks + c] = (hi - lo) * 54;
        }
    }
    /* streams in (row, chunk) order are contiguous in the [kappa][m][54] layout */
    or_chacha8_sample(seeds, (uint32_t)(kappa * n_chunks), counts, Q, out);
    free(seeds); free(counts); free(rows);
}

static uint64_t P2_RCE[8][8], P2_RCI[22], P2_MU[8];
static int p2_ready = 0;
static void p2_init(void) {
    if (p2_ready) return;
    const char* seed = "neo_poseidon2_goldilocks_seed___";
    or_chacha c;
    for (int i = 0; i < 8; i++)
        c.key[i] = (uint32_t)(uint8_t)seed[4*i] | ((uint32_t)(uint8_t)seed[4*i+1] << 8) |
                   ((uint32_t)(uint8_t)seed[4*i+2] << 16) | ((uint32_t)(uint8_t)seed[4*i+3] << 24);
    c.ctr = 0; c.idx = 16;
    uint64_t* outs[3] = {&P2_RCE[0][0], P2_RCI, P2_MU};
    int lens[3] = {64, 22, 8};
    for (int g = 0; g < 3; g++)
        for (int i = 0; i < lens[g]; i++) {
            uint64_t x;
            do { x = cc_u64(&c); } while (x >= Q);
            outs[g][i] = x;
        }
    p2_ready = 1;
}
static uint64_t p2_s7(uint64_t x) { uint64_t x2 = fq_mul(x, x), x3 = fq_mul(x2, x), x6 = fq_mul(x3, x3); return fq_mul(x6, x); }
static void p2_ext(uint64_t* st) {
    static const uint64_t M[4][4] = {{5,7,1,3},{4,6,1,1},{1,3,5,7},{1,1,4,6}};
    uint64_t y[8];
    for (int b = 0; b < 2; b++)
        for (int r = 0; r < 4; r++) {
            uint64_t a = 0;
            for (int cc = 0; cc < 4; cc++) a = fq_add(a, fq_mul(M[r][cc], st[4*b + cc]));
            y[4*b + r] = a;
        }
    for (int i = 0; i < 4; i++) {
        uint64_t s = fq_add(y[i], y[4 + i]);
        st[i] = fq_add(y[i], s);
        st[4 + i] = fq_add(y[4 + i], s);
    }
}
void or_poseidon2_permute(uint64_t* st) {
    p2_init();
    p2_ext(st);
    for (int r = 0; r < 4; r++) { for (int i = 0; i < 8; i++) st[i] = p2_s7(fq_add(st[i], P2_RCE[r][i])); p2_ext(st); }
    for (int r = 0; r < 22; r++) {
        st[0] = p2_s7(fq_add(st[0], P2_RCI[r]));
        uint64_t s = 0;
        for (int i = 0; i < 8; i++) s = fq_add(s, st[i]);
        for (int i = 0; i < 8; i++) st[i] = fq_add(s, fq_mul(P2_MU[i], st[i]));
    }
    for (int r = 4; r < 8; r++) { for (int i = 0; i < 8; i++) st[i] = p2_s7(fq_add(st[i], P2_RCE[r][i])); p2_ext(st); }
}

typedef struct or_transcript { uint64_t st[8]; int absorbed; } or_transcript;
static void tr_perm(or_transcript* t) { or_poseidon2_permute(t->st); t->absorbed = 0; }
static void tr_elem(or_transcript* t, uint64_t x) { if (t->absorbed >= 4) tr_perm(t); t->st[t->absorbed++] = x; }
static void tr_bytes(or_transcript* t, const char* s, size_t n) { for (size_t i = 0; i < n; i++) tr_elem(t, (uint8_t)s[i]); }
void or_tr_append_message(or_transcript* t, const char* label, const uint8_t* msg, size_t len) {
    tr_bytes(t, label, strlen(label));
    tr_elem(t, len);
    for (size_t i = 0; i < len; i++) tr_elem(t, msg[i]);
}
or_transcript* or_tr_new(const char* app_label) {
    or_transcript* t = (or_transcript*)calloc(1, sizeof(*t));
    or_tr_append_message(t, "neo/transcript/v1|poseidon2-goldilocks-w8-r4", (const uint8_t*)app_label, strlen(app_label));
    return t;
}
void or_tr_free(or_transcript* t) { free(t); }
/* Poseidon2Transcript is Clone: fork() clones the sponge (neo-transcript/src/poseidon2.rs:160-164) */
or_transcript* or_tr_clone(const or_transcript* t) {
    or_transcript* c = (or_transcript*)malloc(sizeof(*c));
    memcpy(c, t, sizeof(*c));
    return c;
}
void or_tr_append_fields(or_transcript* t, const char* label, const uint64_t* fs, size_t n) {
    tr_bytes(t, label, strlen(label));
    tr_elem(t, n);
    /* absorb_slice overwrite semantics are element-wise identical to repeated absorb_elem
       except that a full chunk triggers the permutation eagerly (poseidon2.rs:29-60) */
    size_t src = 0;
    while (t->absorbed < 4 && src < n) t->st[t->absorbed++] = fs[src++];
    if (t->absorbed == 4) tr_perm(t);
    while (n - src >= 4) { for (int i = 0; i < 4; i++) t->st[i] = fs[src + i]; tr_perm(t); src += 4; }
    while (src < n) t->st[t->absorbed++] = fs[src++];
}
void or_tr_append_u64s(or_transcript* t, const char* label, const uint64_t* us, size_t n) {
    tr_bytes(t, label, strlen(label));
    tr_elem(t, n);
    for (size_t i = 0; i < n; i++) tr_elem(t, fq_canon(us[i]));
}
uint64_t or_tr_challenge_field(or_transcript* t, const char* label) {
    or_tr_append_message(t, "chal/label", (const uint8_t*)label, strlen(label));
    tr_elem(t, 1);
    tr_perm(t);
    return t->st[0];
}
void or_tr_challenge_fields(or_transcript* t, const char* label, size_t n, uint64_t* out) {
    or_tr_append_message(t, "chal/label", (const uint8_t*)label, strlen(label));
    size_t got = 0;
    while (got < n) { tr_elem(t, 1); tr_perm(t); for (int i = 0; i < 4 && got < n; i++) out[got++] = t->st[i]; }
}
void or_tr_digest32(or_transcript* t, uint8_t* out) {
    tr_elem(t, 1);
    tr_perm(t);
    for (int i = 0; i < 4; i++) for (int b = 0; b < 8; b++) out[8*i + b] = (uint8_t)(t->st[i] >> (8*b));
}
void or_tr_state(const or_transcript* t, uint64_t* out) { memcpy(out, t->st, 64); }

/* Width-16 Poseidon2 for the CCS matrix digest (engines/utils.rs:214-321):
   constants from ChaCha8 seeded by rand_core's seed_from_u64 (PCG32 XSH-RR
   expansion) of 0x434353445F4D4154.  Parity unpinned. */
static uint64_t P16_RCE[8][16], P16_RCI[22], P16_MU[16];
static int p16_ready = 0;
static void p16_init(void) {
    if (p16_ready) return;
    uint8_t seed[32];
    uint64_t state = 0x434353445F4D4154ULL;
    for (int c = 0; c < 8; c++) {
        state = state * 6364136223846793005ULL + 11634580027462260723ULL;
        uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        uint32_t x = (xs >> rot) | (xs << ((32 - rot) & 31));
        for (int b = 0; b < 4; b++) seed[4 * c + b] = (uint8_t)(x >> (8 * b));
    }
    or_chacha c;
    for (int i = 0; i < 8; i++)
        c.key[i] = (uint32_t)seed[4*i] | ((uint32_t)seed[4*i+1] << 8) | ((uint32_t)seed[4*i+2] << 16) | ((uint32_t)seed[4*i+3] << 24);
    c.ctr = 0; c.idx = 16;
    uint64_t* outs[3] = {&P16_RCE[0][0], P16_RCI, P16_MU};
    int lens[3] = {128, 22, 16};
    for (int g = 0; g < 3; g++)
        for (int i = 0; i < lens[g]; i++) {
            uint64_t x;
            do { x = cc_u64(&c); } while (x >= Q);
            outs[g][i] = x;
        }
    p16_ready = 1;
}
static void p16_ext(uint64_t* st) {
    static const uint64_t M[4][4] = {{5,7,1,3},{4,6,1,1},{1,3,5,7},{1,1,4,6}};
    uint64_t y[16];
    for (int b = 0; b < 4; b++)
        for (int r = 0; r < 4; r++) {
            uint64_t a = 0;
            for (int cc = 0; cc < 4; cc++) a = fq_add(a, fq_mul(M[r][cc], st[4*b + cc]));
            y[4*b + r] = a;
        }
    for (int i = 0; i < 4; i++) {
        uint64_t s = 0;
        for (int b = 0; b < 4; b++) s = fq_add(s, y[4*b + i]);
        for (int b = 0; b < 4; b++) st[4*b + i] = fq_add(y[4*b + i], s);
    }
}
void or_poseidon2_w16_permute(uint64_t* st) {
    p16_init();
    p16_ext(st);
    for (int r = 0; r < 4; r++) { for (int i = 0; i < 16; i++) st[i] = p2_s7(fq_add(st[i], P16_RCE[r][i])); p16_ext(st); }
    for (int r = 0; r < 22; r++) {
        st[0] = p2_s7(fq_add(st[0], P16_RCI[r]));
        uint64_t s = 0;
        for (int i = 0; i < 16; i++) s = fq_add(s, st[i]);
        for (int i = 0; i < 16; i++) st[i] = fq_add(s, fq_mul(P16_MU[i], st[i]));
    }
    for (int r = 4; r < 8; r++) { for (int i = 0; i < 16; i++) st[i] = p2_s7(fq_add(st[i], P16_RCE[r][i])); p16_ext(st); }
}

/* digest_ccs_matrices (engines/utils.rs:214-321): dense row-major scan of
   nonzeros, emitted as (row, col, val) triples into a width-16 state. */
void or_ccs_digest(const or_ccs* s, uint64_t* out4) {
    uint64_t st[16] = {0};
    int ab = 0;
    const char* dom = "neo/ccs/matrices/v1";
    for (const char* p = dom; *p; p++) { if (ab >= 15) { or_poseidon2_w16_permute(st); ab = 0; } st[ab++] = (uint8_t)*p; }
    if (ab + 3 >= 16) { or_poseidon2_w16_permute(st); ab = 0; }
    st[ab] = s->n; st[ab + 1] = s->m; st[ab + 2] = s->t;
    or_poseidon2_w16_permute(st);
    for (uint32_t j = 0; j < s->t; j++) {
        ab = 0;
        st[ab++] = j;
        for (uint32_t row = 0; row < s->n; row++) {
            if (s->is_identity[j]) {
                if (ab + 3 > 15) { or_poseidon2_w16_permute(st); ab = 0; }
                st[ab] = row; st[ab + 1] = row; st[ab + 2] = 1; ab += 3;
                continue;
            }
            /* columns ascending within the row: scan the row's entries */
            const uint64_t* cp = s->col_ptr + (size_t)j * (s->m + 1);
            const uint32_t* ri = s->row_idx + s->nnz_off[j];
            const uint64_t* vv = s->vals + s->nnz_off[j];
            (void)cp; (void)ri; (void)vv;
        }
        if (!s->is_identity[j]) {
            /* build row lists (O(nnz)) */
            const uint64_t* cp = s->col_ptr + (size_t)j * (s->m + 1);
            const uint32_t* ri = s->row_idx + s->nnz_off[j];
            const uint64_t* vv = s->vals + s->nnz_off[j];
            uint64_t nnz = s->nnz_off[j + 1] - s->nnz_off[j];
            uint64_t* cnt = (uint64_t*)calloc(s->n + 1, 8);
            for (uint64_t k = 0; k < nnz; k++) cnt[ri[k] + 1]++;
            for (uint32_t r = 0; r < s->n; r++) cnt[r + 1] += cnt[r];
            uint64_t* pos = (uint64_t*)malloc(8 * (s->n + 1));
            memcpy(pos, cnt, 8 * (s->n + 1));
            uint64_t* ec = (uint64_t*)malloc(8 * (nnz ? nnz : 1));
            uint64_t* ev = (uint64_t*)malloc(8 * (nnz ? nnz : 1));
            for (uint32_t c = 0; c < s->m; c++)
                for (uint64_t k = cp[c]; k < cp[c + 1]; k++) { uint64_t p = pos[ri[k]]++; ec[p] = c; ev[p] = vv[k]; }
            for (uint32_t r = 0; r < s->n; r++)
                for (uint64_t e = cnt[r]; e < cnt[r + 1]; e++) {
                    if (ab + 3 > 15) { or_poseidon2_w16_permute(st); ab = 0; }
                    st[ab] = r; st[ab + 1] = ec[e]; st[ab + 2] = fq_canon(ev[e]); ab += 3;
                }
            free(cnt); free(pos); free(ec); free(ev);
        }
        or_poseidon2_w16_permute(st);
    }
    memcpy(out4, st, 32);
}

/* ------------------------------------------------------------------------ */
/* Twist / Shout time-lane oracles (crates/neo-memory/src/twist_oracle.rs).  */
/* This is the literal sparse algorithm: SparseIdxVec columns folded on the  */
/* least-significant bit (sparse_time.rs:69-117), pairs gathered from the    */
/* gate column's entries (twist_oracle.rs:187-199), χ_{r_cycle} children per */
/* pair (twist_oracle.rs:163-185), and Val_pre recomputed at every child     */
/* time point from the increment terms through LT (twist_oracle.rs:311-379). */
/* ------------------------------------------------------------------------ */
typedef struct { size_t len, n; size_t* idx; kq* val; } spv;

static spv spv_from_dense(const kq* d, size_t len) {
    spv v; v.len = len; v.n = 0;
    v.idx = (size_t*)malloc(sizeof(size_t) * (len ? len : 1));
    v.val = (kq*)malloc(sizeof(kq) * (len ? len : 1));
    for (size_t i = 0; i < len; i++) if (!kiszero(d[i])) { v.idx[v.n] = i; v.val[v.n] = d[i]; v.n++; }
    return v;
}
static void spv_free(spv* v) { free(v->idx); free(v->val); }
/* SparseIdxVec::get: binary search, zero when absent (sparse_time.rs:58-64) */
static kq spv_get(const spv* v, size_t i) {
    size_t lo = 0, hi = v->n;
    while (lo < hi) { size_t mid = (lo + hi) / 2; if (v->idx[mid] < i) lo = mid + 1; else hi = mid; }
    return (lo < v->n && v->idx[lo] == i) ? v->val[lo] : K0;
}
static kq spv_single(const spv* v) { return v->n ? v->val[0] : K0; }
/* SparseIdxVec::fold_round_in_place (sparse_time.rs:69-117) */
static void spv_fold(spv* v, kq r) {
    kq omr = ksub(K1, r);
    size_t o = 0, i = 0;
    size_t* nidx = (size_t*)malloc(sizeof(size_t) * (v->n ? v->n : 1));
    kq* nval = (kq*)malloc(sizeof(kq) * (v->n ? v->n : 1));
    while (i < v->n) {
        size_t idx = v->idx[i], parent = idx >> 1;
        kq acc = K0;
        if ((idx & 1) == 0) {
            acc = kadd(acc, kmul(v->val[i], omr)); i++;
            if (i < v->n && v->idx[i] == idx + 1) { acc = kadd(acc, kmul(v->val[i], r)); i++; }
        } else { acc = kadd(acc, kmul(v->val[i], r)); i++; }
        if (!kiszero(acc)) {
            if (o > 0 && nidx[o - 1] == parent) nval[o - 1] = kadd(nval[o - 1], acc);
            else { nidx[o] = parent; nval[o] = acc; o++; }
        }
    }
    free(v->idx); free(v->val);
    v->idx = nidx; v->val = nval; v->n = o; v->len >>= 1;
}

/* eq(bit, u) = bit·(2u − 1) + (1 − u)  (neo-memory/src/bit_ops.rs:5-9) */
static inline kq eq_bit_affine_k(kq bit, kq u) { return kadd(kmul(bit, ksub(kadd(u, u), K1)), ksub(K1, u)); }
static inline kq interp_k(kq f0, kq f1, kq x) { return kadd(f0, kmul(ksub(f1, f0), x)); }

/* twist_oracle.rs:163-185 */
static void chi_cycle_children(const kq* r_cycle, int ell, int bit_idx, kq prefix_eq, size_t pair, kq* c0, kq* c1) {
    kq suffix = K1;
    int shift = 0;
    for (int b = bit_idx + 1; b < ell; b++) {
        suffix = kmul(suffix, ((pair >> shift) & 1) ? r_cycle[b] : ksub(K1, r_cycle[b]));
        shift++;
    }
    kq r = r_cycle[bit_idx];
    *c0 = kmul(kmul(prefix_eq, ksub(K1, r)), suffix);
    *c1 = kmul(kmul(prefix_eq, r), suffix);
}
/* twist_oracle.rs:305-318 */
static void fill_time_point(kq* out, int ell, const kq* prefix, int bit_idx, kq bit_value, size_t pair) {
    for (int b = 0; b < bit_idx; b++) out[b] = prefix[b];
    out[bit_idx] = bit_value;
    int shift = 0;
    for (int b = bit_idx + 1; b < ell; b++) { out[b] = ((pair >> shift) & 1) ? K1 : K0; shift++; }
}
/* LT(idx, point) with idx Boolean (twist_oracle.rs:320-334) */
static kq lt_eval_at_bool_index(size_t idx, const kq* point, int ell) {
    kq suffix = K1, acc = K0;
    for (int i = ell - 1; i >= 0; i--) {
        if (((idx >> i) & 1) == 0) { acc = kadd(acc, kmul(point[i], suffix)); suffix = kmul(suffix, ksub(K1, point[i])); }
        else suffix = kmul(suffix, point[i]);
    }
    return acc;
}
/* LT(j', j) (neo-memory/src/mle.rs:7-24) */
static kq lt_eval_k(const kq* jp, const kq* j, int ell) {
    kq* suf = (kq*)malloc(sizeof(kq) * (ell + 1));
    suf[ell] = K1;
    for (int i = ell - 1; i >= 0; i--) suf[i] = kmul(suf[i + 1], eq_lin(jp[i], j[i]));
    kq acc = K0;
    for (int i = 0; i < ell; i++) acc = kadd(acc, kmul(kmul(ksub(K1, jp[i]), j[i]), suf[i + 1]));
    free(suf);
    return acc;
}

struct or_mem_oracle {
    int kind, ell, ell_addr, bit_idx, degree, n_cols, n_fold;
    kq *rpt, *r_addr, *w, *chal, init, prefix_eq, claim;
    spv* cols;
    size_t n_inc; size_t* inc_t; kq* inc_v;
    kq *t0, *t1;
};

/* build_inc_terms_at_r_addr (twist_oracle.rs:351-378) */
static void build_inc_terms(or_mem_oracle* o, const spv* has_w, const spv* inc, const spv* wa) {
    o->inc_t = (size_t*)malloc(sizeof(size_t) * (has_w->n + 1));
    o->inc_v = (kq*)malloc(sizeof(kq) * (has_w->n + 1));
    o->n_inc = 0;
    for (size_t e = 0; e < has_w->n; e++) {
        size_t t = has_w->idx[e];
        kq hw = has_w->val[e], it = spv_get(inc, t);
        if (kiszero(hw) || kiszero(it)) continue;
        kq eq = K1;
        for (int b = 0; b < o->ell_addr; b++) eq = kmul(eq, eq_bit_affine_k(spv_get(&wa[b], t), o->r_addr[b]));
        kq v = kmul(kmul(hw, it), eq);
        if (!kiszero(v)) { o->inc_t[o->n_inc] = t; o->inc_v[o->n_inc] = v; o->n_inc++; }
    }
}
/* val_pre_from_inc_terms (twist_oracle.rs:336-342) */
static kq val_pre(const or_mem_oracle* o, const kq* tp) {
    kq acc = o->init;
    for (size_t i = 0; i < o->n_inc; i++) acc = kadd(acc, kmul(o->inc_v[i], lt_eval_at_bool_index(o->inc_t[i], tp, o->ell)));
    return acc;
}
static kq eq_addr_at(const or_mem_oracle* o, const spv* bits, size_t t, int single) {
    kq eq = K1;
    for (int b = 0; b < o->ell_addr; b++)
        eq = kmul(eq, eq_bit_affine_k(single ? spv_single(&bits[b]) : spv_get(&bits[b], t), o->r_addr[b]));
    return eq;
}

static int sz_cmp(const void* a, const void* b) {
    size_t x = *(const size_t*)a, y = *(const size_t*)b;
    return x < y ? -1 : x > y;
}

/* Round evaluations at xs (each kind's evals_at). */
static void mem_evals(or_mem_oracle* o, const kq* xs, int nx, kq* ys) {
    int A = o->ell_addr, k = o->kind;
    for (int i = 0; i < nx; i++) ys[i] = K0;
    if (k == OR_MEM_BITNESS && o->n_cols == 0) return;
    if (o->cols[0].len == 1) {
        kq v = K0;
        switch (k) {
            case OR_MEM_SHOUT_VALUE: v = kmul(kmul(o->prefix_eq, spv_single(&o->cols[0])), spv_single(&o->cols[1])); break;
            case OR_MEM_SHOUT_ADAPTER: v = kmul(kmul(o->prefix_eq, spv_single(&o->cols[0])), eq_addr_at(o, &o->cols[1], 0, 1)); break;
            case OR_MEM_BITNESS: {
                kq acc = K0;
                for (int c = 0; c < o->n_cols; c++) { kq b = spv_single(&o->cols[c]); acc = kadd(acc, kmul(kmul(o->w[c], b), ksub(b, K1))); }
                v = kmul(o->prefix_eq, acc);
            } break;
            case OR_MEM_TWIST_READ: {
                kq diff = ksub(val_pre(o, o->chal), spv_single(&o->cols[1]));
                v = kmul(kmul(kmul(o->prefix_eq, spv_single(&o->cols[0])), diff), eq_addr_at(o, &o->cols[2], 0, 1));
            } break;
            case OR_MEM_TWIST_WRITE: {
                kq delta = ksub(ksub(spv_single(&o->cols[1]), val_pre(o, o->chal)), spv_single(&o->cols[2]));
                v = kmul(kmul(kmul(o->prefix_eq, spv_single(&o->cols[0])), delta), eq_addr_at(o, &o->cols[3], 0, 1));
            } break;
            case OR_MEM_VAL_EVAL:
                v = kmul(kmul(kmul(spv_single(&o->cols[0]), spv_single(&o->cols[1])), eq_addr_at(o, &o->cols[2], 0, 1)),
                         lt_eval_k(o->chal, o->rpt, o->ell));
                break;
            case OR_MEM_TOTAL_INC:
                v = kmul(kmul(spv_single(&o->cols[0]), spv_single(&o->cols[1])), eq_addr_at(o, &o->cols[2], 0, 1));
                break;
            case OR_MEM_PRODUCT: {
                v = K1;
                for (int c = 0; c < o->n_cols; c++) v = kmul(v, spv_single(&o->cols[c]));
            } break;
        }
        for (int i = 0; i < nx; i++) ys[i] = v;
        return;
    }
    /* pairs: from the gate column (gather_pairs_from_sparse), the union of all
       columns for bitness (twist_oracle.rs:560-568), every pair for products */
    size_t np = 0, half = o->cols[0].len / 2;
    size_t* pairs;
    if (k == OR_MEM_PRODUCT) {
        pairs = (size_t*)malloc(sizeof(size_t) * half);
        for (size_t p = 0; p < half; p++) pairs[np++] = p;
    } else if (k == OR_MEM_BITNESS) {
        size_t tot = 0;
        for (int c = 0; c < o->n_cols; c++) tot += o->cols[c].n;
        pairs = (size_t*)malloc(sizeof(size_t) * (tot + 1));
        for (int c = 0; c < o->n_cols; c++) for (size_t e = 0; e < o->cols[c].n; e++) pairs[np++] = o->cols[c].idx[e] >> 1;
        qsort(pairs, np, sizeof(size_t), sz_cmp);
        size_t u = 0;
        for (size_t i = 0; i < np; i++) if (u == 0 || pairs[u - 1] != pairs[i]) pairs[u++] = pairs[i];
        np = u;
    } else {
        pairs = (size_t*)malloc(sizeof(size_t) * (o->cols[0].n + 1));
        for (size_t e = 0; e < o->cols[0].n; e++) {
            size_t p = o->cols[0].idx[e] >> 1;
            if (np == 0 || pairs[np - 1] != p) pairs[np++] = p;
        }
    }
    int maxf = 4 + A + o->n_cols;
    kq* f0 = (kq*)malloc(sizeof(kq) * maxf);
    kq* f1 = (kq*)malloc(sizeof(kq) * maxf);
    for (size_t pi = 0; pi < np; pi++) {
        size_t pair = pairs[pi], c0 = 2 * pair, c1 = c0 + 1;
        int nf = 0;
        if (k == OR_MEM_BITNESS) {
            kq ch0, ch1;
            chi_cycle_children(o->rpt, o->ell, o->bit_idx, o->prefix_eq, pair, &ch0, &ch1);
            for (int i = 0; i < nx; i++) {
                kq chi_x = interp_k(ch0, ch1, xs[i]);
                if (kiszero(chi_x)) continue;
                kq bs = K0;
                for (int c = 0; c < o->n_cols; c++) {
                    kq b0 = spv_get(&o->cols[c], c0), b1 = spv_get(&o->cols[c], c1);
                    if (kiszero(b0) && kiszero(b1)) continue;
                    kq bx = interp_k(b0, b1, xs[i]);
                    bs = kadd(bs, kmul(kmul(o->w[c], bx), ksub(bx, K1)));
                }
                ys[i] = kadd(ys[i], kmul(chi_x, bs));
            }
            continue;
        }
        if (k != OR_MEM_PRODUCT) {
            kq g0 = spv_get(&o->cols[0], c0), g1 = spv_get(&o->cols[0], c1);
            if (kiszero(g0) && kiszero(g1)) continue;
            f0[nf] = g0; f1[nf] = g1; nf++;
        }
        if (k == OR_MEM_SHOUT_VALUE || k == OR_MEM_SHOUT_ADAPTER || k == OR_MEM_TWIST_READ || k == OR_MEM_TWIST_WRITE) {
            chi_cycle_children(o->rpt, o->ell, o->bit_idx, o->prefix_eq, pair, &f0[nf], &f1[nf]); nf++;
        }
        const spv* bits = NULL;
        switch (k) {
            case OR_MEM_SHOUT_VALUE:
                f0[nf] = spv_get(&o->cols[1], c0); f1[nf] = spv_get(&o->cols[1], c1); nf++;
                break;
            case OR_MEM_SHOUT_ADAPTER: bits = &o->cols[1]; break;
            case OR_MEM_TWIST_READ: {
                fill_time_point(o->t0, o->ell, o->chal, o->bit_idx, K0, pair);
                fill_time_point(o->t1, o->ell, o->chal, o->bit_idx, K1, pair);
                f0[nf] = ksub(val_pre(o, o->t0), spv_get(&o->cols[1], c0));
                f1[nf] = ksub(val_pre(o, o->t1), spv_get(&o->cols[1], c1)); nf++;
                bits = &o->cols[2];
            } break;
            case OR_MEM_TWIST_WRITE: {
                fill_time_point(o->t0, o->ell, o->chal, o->bit_idx, K0, pair);
                fill_time_point(o->t1, o->ell, o->chal, o->bit_idx, K1, pair);
                f0[nf] = ksub(ksub(spv_get(&o->cols[1], c0), val_pre(o, o->t0)), spv_get(&o->cols[2], c0));
                f1[nf] = ksub(ksub(spv_get(&o->cols[1], c1), val_pre(o, o->t1)), spv_get(&o->cols[2], c1)); nf++;
                bits = &o->cols[3];
            } break;
            case OR_MEM_VAL_EVAL: {
                f0[nf] = spv_get(&o->cols[1], c0); f1[nf] = spv_get(&o->cols[1], c1); nf++;
                fill_time_point(o->t0, o->ell, o->chal, o->bit_idx, K0, pair);
                fill_time_point(o->t1, o->ell, o->chal, o->bit_idx, K1, pair);
                f0[nf] = lt_eval_k(o->t0, o->rpt, o->ell); f1[nf] = lt_eval_k(o->t1, o->rpt, o->ell); nf++;
                bits = &o->cols[2];
            } break;
            case OR_MEM_TOTAL_INC:
                f0[nf] = spv_get(&o->cols[1], c0); f1[nf] = spv_get(&o->cols[1], c1); nf++;
                bits = &o->cols[2];
                break;
            case OR_MEM_PRODUCT:
                for (int c = 0; c < o->n_cols; c++) { f0[nf] = spv_get(&o->cols[c], c0); f1[nf] = spv_get(&o->cols[c], c1); nf++; }
                break;
        }
        if (bits)
            for (int b = 0; b < A; b++) {
                f0[nf] = eq_bit_affine_k(spv_get(&bits[b], c0), o->r_addr[b]);
                f1[nf] = eq_bit_affine_k(spv_get(&bits[b], c1), o->r_addr[b]);
                nf++;
            }
        for (int i = 0; i < nx; i++) {
            kq prod = K1;
            for (int f = 0; f < nf; f++) prod = kmul(prod, interp_k(f0[f], f1[f], xs[i]));
            ys[i] = kadd(ys[i], prod);
        }
    }
    free(f0); free(f1); free(pairs);
}

or_mem_oracle* or_mem_oracle_new(int kind, int ell, const uint64_t* r_point, int ell_addr, const uint64_t* r_addr,
                                 const uint64_t* init, int n_cols, const uint64_t* cols, const uint64_t* weights,
                                 uint64_t* claim_out) {
    int A = ell_addr;
    int need = -1;
    switch (kind) {
        case OR_MEM_SHOUT_VALUE: need = 2; break;
        case OR_MEM_SHOUT_ADAPTER: need = 1 + A; break;
        case OR_MEM_BITNESS: need = n_cols; break;
        case OR_MEM_TWIST_READ: need = 4 + 2 * A; break;
        case OR_MEM_TWIST_WRITE: need = 3 + A; break;
        case OR_MEM_VAL_EVAL: case OR_MEM_TOTAL_INC: need = 2 + A; break;
        case OR_MEM_PRODUCT: need = n_cols; break;
        default: return NULL;
    }
    if (n_cols != need || ell < 0) return NULL;
    or_mem_oracle* o = (or_mem_oracle*)calloc(1, sizeof(*o));
    size_t L = (size_t)1 << ell;
    o->kind = kind; o->ell = ell; o->ell_addr = A; o->n_cols = n_cols;
    o->rpt = kdup(r_point, r_point ? ell : 0);
    o->r_addr = kdup(r_addr, r_addr ? A : 0);
    o->init = init ? kload(init) : K0;
    o->prefix_eq = K1;
    o->chal = (kq*)calloc(ell + 1, sizeof(kq));
    o->t0 = (kq*)calloc(ell + 1, sizeof(kq));
    o->t1 = (kq*)calloc(ell + 1, sizeof(kq));
    o->cols = (spv*)calloc(n_cols + 1, sizeof(spv));
    for (int c = 0; c < n_cols; c++) o->cols[c] = spv_from_dense((const kq*)cols + (size_t)c * L, L);
    if (kind == OR_MEM_BITNESS) o->w = kdup(weights, n_cols);
    o->n_fold = n_cols;
    switch (kind) {
        case OR_MEM_SHOUT_VALUE: case OR_MEM_BITNESS: o->degree = 3; break;
        case OR_MEM_SHOUT_ADAPTER: o->degree = 2 + A; break;
        case OR_MEM_TWIST_READ:
            o->degree = 3 + A; o->n_fold = 2 + A;  /* the write stream enters only through Val_pre */
            build_inc_terms(o, &o->cols[2 + A], &o->cols[3 + A], &o->cols[4 + A]);
            break;
        case OR_MEM_TWIST_WRITE:
            o->degree = 3 + A;
            build_inc_terms(o, &o->cols[0], &o->cols[2], &o->cols[3]);
            break;
        case OR_MEM_VAL_EVAL: o->degree = 3 + A; break;
        case OR_MEM_TOTAL_INC: o->degree = 2 + A; break;
        case OR_MEM_PRODUCT: o->degree = n_cols; break;
    }
    /* claims: the constructors' direct sums where the reference computes one
       (twist_oracle.rs:214-241, 396-437, 928-974, 1064-1102, 89-101); the
       hypercube sum p(0) + p(1) of round 0 for bitness / read / write checks,
       whose claimed sums the caller supplies (zero for an honest witness) */
    kq claim = K0;
    if (kind == OR_MEM_SHOUT_VALUE) {
        for (size_t e = 0; e < o->cols[0].n; e++) {
            size_t t = o->cols[0].idx[e];
            kq v = spv_get(&o->cols[1], t);
            if (kiszero(v)) continue;
            claim = kadd(claim, kmul(kmul(eq_points_bool_mask(t, o->rpt, ell), o->cols[0].val[e]), v));
        }
    } else if (kind == OR_MEM_SHOUT_ADAPTER) {
        for (size_t e = 0; e < o->cols[0].n; e++) {
            size_t t = o->cols[0].idx[e];
            claim = kadd(claim, kmul(kmul(eq_points_bool_mask(t, o->rpt, ell), o->cols[0].val[e]), eq_addr_at(o, &o->cols[1], t, 0)));
        }
    } else if (kind == OR_MEM_VAL_EVAL || kind == OR_MEM_TOTAL_INC) {
        for (size_t e = 0; e < o->cols[0].n; e++) {
            size_t t = o->cols[0].idx[e];
            kq it = spv_get(&o->cols[1], t);
            if (kiszero(it)) continue;
            kq term = kmul(kmul(o->cols[0].val[e], it), eq_addr_at(o, &o->cols[2], t, 0));
            if (kind == OR_MEM_VAL_EVAL) term = kmul(term, lt_eval_at_bool_index(t, o->rpt, ell));
            claim = kadd(claim, term);
        }
    } else if (kind == OR_MEM_PRODUCT) {
        for (size_t t = 0; t < L; t++) {
            kq p = K1;
            for (int c = 0; c < n_cols; c++) p = kmul(p, ((const kq*)cols)[(size_t)c * L + t]);
            claim = kadd(claim, p);
        }
    } else if (ell > 0) {
        kq xs[2] = {K0, K1}, ys[2];
        mem_evals(o, xs, 2, ys);
        claim = kadd(ys[0], ys[1]);
    } else {
        kq xs[1] = {K0}, ys[1];
        mem_evals(o, xs, 1, ys);
        claim = ys[0];
    }
    o->claim = claim;
    if (claim_out) kstore(claim_out, claim);
    return o;
}

void or_mem_oracle_free(or_mem_oracle* o) {
    if (!o) return;
    for (int c = 0; c < o->n_cols; c++) spv_free(&o->cols[c]);
    free(o->cols); free(o->rpt); free(o->r_addr); free(o->w); free(o->chal); free(o->t0); free(o->t1);
    free(o->inc_t); free(o->inc_v); free(o);
}
int or_mem_oracle_num_rounds(const or_mem_oracle* o) { return o->ell - o->bit_idx; }
int or_mem_oracle_degree_bound(const or_mem_oracle* o) { return o->degree; }
void or_mem_oracle_evals(or_mem_oracle* o, const uint64_t* xs, int nx, uint64_t* ys) {
    mem_evals(o, (const kq*)xs, nx, (kq*)ys);
}
void or_mem_oracle_fold(or_mem_oracle* o, const uint64_t* rp) {
    if (o->bit_idx >= o->ell) return;
    kq r = kload(rp);
    int k = o->kind;
    if (k == OR_MEM_SHOUT_VALUE || k == OR_MEM_SHOUT_ADAPTER || k == OR_MEM_BITNESS || k == OR_MEM_TWIST_READ ||
        k == OR_MEM_TWIST_WRITE)
        o->prefix_eq = kmul(o->prefix_eq, eq_lin(r, o->rpt[o->bit_idx]));
    for (int c = 0; c < o->n_fold; c++) spv_fold(&o->cols[c], r);
    o->chal[o->bit_idx++] = r;
}

/* Weight table of AddressLookupOracle::new (twist_oracle.rs:1671-1724):
   w[addr(t)] += χ_{r_cycle}(t)·has_lookup(t), addr(t) from bit columns equal
   to one; claim = Σ_a table[a]·w[a]. */
void or_addr_lookup_weights(int ell, const uint64_t* r_cycle, int ell_addr, const uint64_t* has_lookup,
                            const uint64_t* addr_bits, const uint64_t* table, size_t table_len,
                            uint64_t* weights_out, uint64_t* claim_out) {
    size_t L = (size_t)1 << ell, P = (size_t)1 << ell_addr;
    kq* r = kdup(r_cycle, ell);
    kq* w = (kq*)weights_out;
    for (size_t a = 0; a < P; a++) w[a] = K0;
    const kq* hl = (const kq*)has_lookup;
    const kq* ab = (const kq*)addr_bits;
    for (size_t t = 0; t < L; t++) {
        if (kiszero(hl[t])) continue;
        kq wt = kmul(eq_points_bool_mask(t, r, ell), hl[t]);
        if (kiszero(wt)) continue;
        size_t a = 0;
        for (int b = 0; b < ell_addr; b++) if (keq(ab[(size_t)b * L + t], K1)) a |= (size_t)1 << b;
        w[a] = kadd(w[a], wt);
    }
    kq claim = K0;
    for (size_t a = 0; a < P && a < table_len; a++) claim = kadd(claim, kmul(((const kq*)table)[a], w[a]));
    kstore(claim_out, claim);
    free(r);
}

/* ------------------------------------------------------------------------ */
/* Twist address-lane oracles: TwistReadCheckAddrOracleSparseTime and        */
/* TwistWriteCheckAddrOracleSparseTime (twist_oracle.rs:1259-1642). Events   */
/* are the merged nonzero times of has_read / has_write (read) or of         */
/* has_write (write); a memory keyed by addr >> bit_idx is replayed in time  */
/* order every round (reads see it before the same event's write).          */
/* ------------------------------------------------------------------------ */
struct or_twist_addr {
    int kind, ell_addr, bit_idx;
    size_t n_ev, n_init;
    kq *eq, *hr, *rv, *hw, *inc, *wv, *rpw, *wpw, *ival, *ipw;
    size_t *ra, *wa, *iaddr;
    kq* mem;
};
typedef struct or_twist_addr or_twist_addr;

/* addr_from_sparse_bits_at_time (twist_oracle.rs:1207-1215): bit b set iff column b equals one */
static size_t addr_at(const kq* bits, size_t L, int A, size_t t) {
    size_t a = 0;
    for (int b = 0; b < A; b++) if (keq(bits[(size_t)b * L + t], K1)) a |= (size_t)1 << b;
    return a;
}

/* kind 0: cols [has_read, rv, ra_bits x A, has_write, inc, wa_bits x A];
   kind 1: cols [has_write, wv, inc, wa_bits x A]. init: n_init (addr, K value). */
or_twist_addr* or_twist_addr_new(int kind, int ell, const uint64_t* r_cycle, int A, size_t n_init,
                                 const uint64_t* init_addr, const uint64_t* init_val, const uint64_t* cols) {
    size_t L = (size_t)1 << ell;
    const kq* C = (const kq*)cols;
    const kq *hr = NULL, *rv = NULL, *ra = NULL, *hw, *inc, *wa, *wv = NULL;
    if (kind == 0) { hr = C; rv = C + L; ra = C + 2 * L; hw = C + (2 + A) * L; inc = C + (3 + A) * L; wa = C + (4 + A) * L; }
    else { hw = C; wv = C + L; inc = C + 2 * L; wa = C + 3 * L; }
    kq* r = kdup(r_cycle, ell);
    or_twist_addr* o = (or_twist_addr*)calloc(1, sizeof(*o));
    o->kind = kind; o->ell_addr = A;
    size_t cap = L ? L : 1;
#define ALLOC_K(f) o->f = (kq*)calloc(cap, sizeof(kq))
    ALLOC_K(eq); ALLOC_K(hr); ALLOC_K(rv); ALLOC_K(hw); ALLOC_K(inc); ALLOC_K(wv); ALLOC_K(rpw); ALLOC_K(wpw);
#undef ALLOC_K
    o->ra = (size_t*)calloc(cap, sizeof(size_t));
    o->wa = (size_t*)calloc(cap, sizeof(size_t));
    size_t n = 0;
    for (size_t t = 0; t < L; t++) {
        int has_r = kind == 0 && !kiszero(hr[t]);
        int has_w = !kiszero(hw[t]);
        if (!has_r && !has_w) continue;
        o->eq[n] = eq_points_bool_mask(t, r, ell);
        o->hw[n] = hw[t];
        o->inc[n] = inc[t];
        if (kind == 0) {
            o->hr[n] = hr[t];
            o->rv[n] = rv[t];
            o->ra[n] = has_r ? addr_at(ra, L, A, t) : 0;
            o->wa[n] = has_w ? addr_at(wa, L, A, t) : 0;
        } else {
            o->wv[n] = wv[t];
            o->wa[n] = addr_at(wa, L, A, t);
        }
        o->rpw[n] = K1;
        o->wpw[n] = K1;
        n++;
    }
    o->n_ev = n;
    o->n_init = n_init;
    o->iaddr = (size_t*)calloc(n_init + 1, sizeof(size_t));
    o->ival = (kq*)calloc(n_init + 1, sizeof(kq));
    o->ipw = (kq*)calloc(n_init + 1, sizeof(kq));
    for (size_t i = 0; i < n_init; i++) { o->iaddr[i] = init_addr[i]; o->ival[i] = kload(init_val + 2 * i); o->ipw[i] = K1; }
    o->mem = (kq*)calloc(((size_t)1 << A) + 1, sizeof(kq));
    free(r);
    return o;
}

void or_twist_addr_free(or_twist_addr* o) {
    if (!o) return;
    free(o->eq); free(o->hr); free(o->rv); free(o->hw); free(o->inc); free(o->wv); free(o->rpw); free(o->wpw);
    free(o->ra); free(o->wa); free(o->iaddr); free(o->ival); free(o->ipw); free(o->mem); free(o);
}
int or_twist_addr_num_rounds(const or_twist_addr* o) { return o->ell_addr - o->bit_idx; }

void or_twist_addr_evals(or_twist_addr* o, const uint64_t* xs_u, int nx, uint64_t* ys_u) {
    const kq* xs = (const kq*)xs_u;
    kq* ys = (kq*)ys_u;
    for (int i = 0; i < nx; i++) ys[i] = K0;
    if (o->bit_idx >= o->ell_addr) {
        kq mem = K0, sum = K0;
        for (size_t i = 0; i < o->n_init; i++) mem = kadd(mem, kmul(o->ival[i], o->ipw[i]));
        for (size_t i = 0; i < o->n_ev; i++) {
            if (o->kind == 0) {
                if (!kiszero(o->hr[i]))
                    sum = kadd(sum, kmul(kmul(kmul(o->eq[i], o->hr[i]), o->rpw[i]), ksub(mem, o->rv[i])));
            } else {
                kq delta = ksub(ksub(o->wv[i], mem), o->inc[i]);
                sum = kadd(sum, kmul(kmul(kmul(o->eq[i], o->hw[i]), o->wpw[i]), delta));
            }
            if (!kiszero(o->hw[i])) mem = kadd(mem, kmul(kmul(o->inc[i], o->hw[i]), o->wpw[i]));
        }
        for (int i = 0; i < nx; i++) ys[i] = sum;
        return;
    }
    const int bit = o->bit_idx;
    const size_t P = (size_t)1 << (o->ell_addr - bit);
    kq* mem = o->mem;
    for (size_t a = 0; a < P; a++) mem[a] = K0;
    for (size_t i = 0; i < o->n_init; i++) mem[o->iaddr[i] >> bit] = kadd(mem[o->iaddr[i] >> bit], kmul(o->ival[i], o->ipw[i]));
    for (size_t i = 0; i < o->n_ev; i++) {
        const int q_read = o->kind == 0 && !kiszero(o->hr[i]);
        const int q_write = o->kind == 1 && !kiszero(o->hw[i]);
        if (q_read || q_write) {
            const size_t a = q_read ? o->ra[i] : o->wa[i];
            const size_t base = (a >> (bit + 1)) * 2;
            const kq v0 = mem[base], v1 = mem[base + 1], dv = ksub(v1, v0);
            const int b = (a >> bit) & 1;
            const kq w = q_read ? kmul(kmul(o->eq[i], o->hr[i]), o->rpw[i]) : kmul(kmul(o->eq[i], o->hw[i]), o->wpw[i]);
            for (int j = 0; j < nx; j++) {
                kq vx = kadd(v0, kmul(dv, xs[j]));
                kq af = b ? xs[j] : ksub(K1, xs[j]);
                kq term = q_read ? ksub(vx, o->rv[i]) : ksub(ksub(o->wv[i], vx), o->inc[i]);
                ys[j] = kadd(ys[j], kmul(kmul(w, af), term));
            }
        }
        if (!kiszero(o->hw[i])) {
            size_t idx = o->wa[i] >> bit;
            mem[idx] = kadd(mem[idx], kmul(kmul(o->inc[i], o->hw[i]), o->wpw[i]));
        }
    }
}

/* update_prefix_weights_in_place (twist_oracle.rs:1196-1205) */
void or_twist_addr_fold(or_twist_addr* o, const uint64_t* rp) {
    if (o->bit_idx >= o->ell_addr) return;
    kq r = kload(rp), omr = ksub(K1, r);
    int bit = o->bit_idx;
    for (size_t i = 0; i < o->n_init; i++) o->ipw[i] = kmul(o->ipw[i], ((o->iaddr[i] >> bit) & 1) ? r : omr);
    for (size_t i = 0; i < o->n_ev; i++) {
        if (o->kind == 0) o->rpw[i] = kmul(o->rpw[i], ((o->ra[i] >> bit) & 1) ? r : omr);
        o->wpw[i] = kmul(o->wpw[i], ((o->wa[i] >> bit) & 1) ? r : omr);
    }
    o->bit_idx++;
}

/* append_bus_openings_to_me_instance (crates/neo-fold/src/memory_sidecar/cpu_bus.rs:195-320):
   y[c][rho] = Σ_j χ_r(m_in + j)·Z[rho][bus_base + col_c·chunk + j], y_scalar[c] = Σ_rho b^rho y[c][rho]. */
void or_bus_openings(const int8_t* Z, int64_t m, int64_t bus_base, int64_t chunk, int n_cols, int64_t m_in,
                     const uint64_t* r, int ell, uint64_t* y_out /* [n_cols][54] K */, uint64_t* ysc_out) {
    kq* rr = kdup(r, ell);
    kq* w = (kq*)malloc(sizeof(kq) * (chunk ? chunk : 1));
    for (int64_t j = 0; j < chunk; j++) w[j] = eq_points_bool_mask((size_t)(m_in + j), rr, ell);
    kq* y = (kq*)y_out;
    for (int c = 0; c < n_cols; c++) {
        kq sc = K0, pw = K1;
        for (int rho = 0; rho < D; rho++) {
            kq acc = K0;
            for (int64_t j = 0; j < chunk; j++) {
                int8_t z = Z[(size_t)rho * m + bus_base + (int64_t)c * chunk + j];
                if (z) acc = kadd(acc, kmul(w[j], kfq(fq_from_i64(z))));
            }
            y[(size_t)c * D + rho] = acc;
            sc = kadd(sc, kmul(acc, pw));
            pw = kscale(pw, 2);
        }
        kstore(ysc_out + 2 * c, sc);
    }
    free(rr); free(w);
}
