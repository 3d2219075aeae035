/*
 * neo_oracle.h -- CPU restatement of Nightstream's Neo fold-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA library (nightstream_b200/csrc) and the timed CPU baseline.  Only the
 * test suite, the smoke check and the CPU-baseline leg of bench.py load it;
 * the product path never calls it.
 *
 * Every routine restates a reference function (path:line is relative to the
 * reference project root, crates/...).  All arithmetic is exact: Fq is the
 * Goldilocks field q = 2^64 - 2^32 + 1 (canonical u64 < q); K = Fq[u]/(u^2-7)
 * stored as two consecutive u64 (re, im); Rq = Fq[X]/(X^54 + X^27 + 1).
 *
 * Parity status: arithmetic, commitment, decomposition, RLC/DEC, Pi_CCS
 * oracle and sum-check driver are pinned by definition and by the
 * reference's relational tests (paper-exact Q, S-homomorphism, round-trip).
 * The Poseidon2 round constants and the ChaCha8 stream used for them come
 * from un-vendored crates (p3-poseidon2 0.4.1, rand_chacha 0.9.0): the
 * transcript here is a restatement of the published designs and its exact
 * states are "parity unpinned".
 */
#ifndef NEO_ORACLE_H
#define NEO_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_D 54
#define OR_Q 0xFFFFFFFF00000001ULL

/* ---- field / ring (neo-math/src/field.rs:10-16, ring.rs:54-67) ---- */
void or_fq_mul_batch(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out);
void or_k_mul_batch(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out);
void or_k_inv_batch(const uint64_t* a, size_t n, uint64_t* out);
void or_rq_mul(const uint64_t* a, const uint64_t* b, uint64_t* out);

/* ---- Ajtai (neo-ajtai/src/commit.rs:679-744, decomp.rs:118-158) ---- */
/* pp: [kappa][m][54] canonical; Z: [54][m] row-major digits; out: [kappa][54] */
void or_commit_digits(const uint64_t* pp, int kappa, int64_t m, const int8_t* Z, uint64_t* out, int threads);
/* general Fq-valued Z (row-major [54][m]) */
void or_commit_fq(const uint64_t* pp, int kappa, int64_t m, const uint64_t* Z, uint64_t* out);
/* z: [m] canonical -> Z [54][m] balanced base-2 digits (values beyond 54 digits drop, as the reference) */
void or_decomp_b2(const uint64_t* z, int64_t m, int8_t* Z);
/* z recomposition: z[c] = sum_rho 2^rho Z[rho][c] mod q */
void or_recompose_b2(const int8_t* Z, int64_t m, uint64_t* z);

/* ---- RLC / DEC (neo-reductions/src/common.rs:75-268, 370-573) ---- */
/* Z_mix[54][m] = sum_i rot(a_i) Z_i with a_i in {-2..2}^54, Z_i in small ints. */
void or_rlc_mix(const int8_t* rho_coeffs, const int8_t* Zs, int count, int64_t m, int32_t* Zmix, int threads);
/* balanced base-b split of small signed Zmix into k planes; returns 0 or -1 (out of range) */
int or_split_b(const int32_t* Zmix, int64_t len, int k, int b, int8_t* planes, uint8_t* nonzero);
/* rot(a) as a dense 54x54 row-major Fq matrix (common.rs:398-430) */
void or_rot_matrix(const int8_t* a, uint64_t* out);

/* ---- sum-check (neo-reductions/src/sumcheck.rs:48-118) ---- */
void or_interpolate(const uint64_t* xs, const uint64_t* ys, int n, uint64_t* coeffs);
void or_poly_eval_k(const uint64_t* coeffs, int n, const uint64_t* x, uint64_t* out);
void or_chi_table(const uint64_t* bits, int nbits, uint64_t* out);

/* ---- CCS description (neo-ccs/src/relations.rs, sparse.rs) ---- */
typedef struct or_ccs {
    uint32_t n, m, t;
    const uint8_t* is_identity;  /* [t] */
    const uint64_t* col_ptr;     /* [t*(m+1)] CSC column pointers, relative to nnz_off[j] */
    const uint64_t* nnz_off;     /* [t+1] */
    const uint32_t* row_idx;     /* [nnz_off[t]] */
    const uint64_t* vals;        /* [nnz_off[t]] canonical */
    uint32_t n_terms;
    const uint64_t* f_coeff;     /* [n_terms] */
    const uint32_t* f_exps;      /* [n_terms*t] */
} or_ccs;

/* ---- Pi_CCS optimized oracle (optimized_engine/oracle.rs:82-503, 1047-1178, 1659-2104) ---- */
typedef struct or_ccs_oracle or_ccs_oracle;
/* Z: [k][54][m] digits (MCS witnesses first, then ME); challenges as K pairs.
   r_inputs may be NULL (step 0). */
or_ccs_oracle* or_ccs_oracle_new(const or_ccs* s, const int8_t* Z, int k, int b,
                                 const uint64_t* alpha, const uint64_t* beta_a, const uint64_t* beta_r,
                                 const uint64_t* gamma, const uint64_t* r_inputs,
                                 int ell_d, int ell_n, int d_sc);
void or_ccs_oracle_free(or_ccs_oracle* o);
int or_ccs_oracle_num_rounds(const or_ccs_oracle* o);
void or_ccs_oracle_evals(or_ccs_oracle* o, const uint64_t* xs, int nx, uint64_t* ys);
void or_ccs_oracle_fold(or_ccs_oracle* o, const uint64_t* r);
/* y_out: [k][t][54] K ; y_scalars: [k][t] K (oracle.rs:1955-2072) */
void or_ccs_oracle_me_outputs(or_ccs_oracle* o, uint64_t* y_out, uint64_t* y_scalars);
/* Run all rounds with externally supplied challenges; writes per-round evals [rounds][d_sc+1] K.
   Returns -1-round on a p(0)+p(1) invariant failure, else 0. */
int or_ccs_sumcheck_fixed(or_ccs_oracle* o, const uint64_t* initial_sum, const uint64_t* chals,
                          uint64_t* evals_out, uint64_t* final_sum);

/* ---- paper-exact Q (paper_exact_engine/paper_exact.rs:236-340, 414-687) ---- */
void or_q_sum_hypercube(const or_ccs* s, const int8_t* Z, int k, int b,
                        const uint64_t* alpha, const uint64_t* beta_a, const uint64_t* beta_r,
                        const uint64_t* gamma, const uint64_t* r_inputs, int ell_d, int ell_n, uint64_t* out);
void or_q_eval_ext(const or_ccs* s, const int8_t* Z, int k, int b,
                   const uint64_t* alpha, const uint64_t* beta_a, const uint64_t* beta_r,
                   const uint64_t* gamma, const uint64_t* r_inputs, int ell_d, int ell_n,
                   const uint64_t* alpha_p, const uint64_t* r_p, uint64_t* out);

/* ---- ME y from Z at point r (common.rs:582-650): y[t][54] K, y_scalars[t] ---- */
void or_me_y_at_r(const or_ccs* s, const int8_t* Z, int ell_n, const uint64_t* r, int b,
                  uint64_t* y, uint64_t* y_scalars);

/* ---- transcript (crates/neo-transcript/src/poseidon2.rs; parity unpinned) ---- */
typedef struct or_transcript or_transcript;
void or_poseidon2_permute(uint64_t* st);
or_transcript* or_tr_new(const char* app_label);
void or_tr_free(or_transcript* t);
or_transcript* or_tr_clone(const or_transcript* t);
void or_tr_append_message(or_transcript* t, const char* label, const uint8_t* msg, size_t len);
void or_tr_append_fields(or_transcript* t, const char* label, const uint64_t* fs, size_t n);
void or_tr_append_u64s(or_transcript* t, const char* label, const uint64_t* us, size_t n);
uint64_t or_tr_challenge_field(or_transcript* t, const char* label);
void or_tr_challenge_fields(or_transcript* t, const char* label, size_t n, uint64_t* out);
void or_tr_digest32(or_transcript* t, uint8_t* out);
void or_tr_state(const or_transcript* t, uint64_t* out);
void or_poseidon2_w16_permute(uint64_t* st);

/* Ajtai PP generation from ChaCha8 (crates/neo-ajtai/src/commit.rs:21-264) */
void or_chacha8_sample(const uint8_t* seeds, uint32_t n_streams, const uint64_t* counts, uint64_t bound,
                       uint64_t* out);
void or_pp_setup(const uint8_t* seed, uint32_t kappa, uint64_t m, int mode, uint64_t* out);
void or_ccs_digest(const or_ccs* s, uint64_t* out4);


/* Twist / Shout time-lane oracles (crates/neo-memory/src/twist_oracle.rs).
   cols: n_cols dense K columns of 2^ell entries; layouts per kind:
   SHOUT_VALUE [has_lookup, val]; SHOUT_ADAPTER [has_lookup, addr_bits...];
   BITNESS [cols...] with weights; TWIST_READ [has_read, rv, ra_bits...,
   has_write, inc_at_write_addr, wa_bits...]; TWIST_WRITE [has_write, wv,
   inc_at_write_addr, wa_bits...]; VAL_EVAL / TOTAL_INC [has_write,
   inc_at_write_addr, wa_bits...]; PRODUCT [factors...]. */
enum { OR_MEM_SHOUT_VALUE = 0, OR_MEM_SHOUT_ADAPTER = 1, OR_MEM_BITNESS = 2, OR_MEM_TWIST_READ = 3,
       OR_MEM_TWIST_WRITE = 4, OR_MEM_VAL_EVAL = 5, OR_MEM_TOTAL_INC = 6, OR_MEM_PRODUCT = 7 };
typedef struct or_mem_oracle or_mem_oracle;
or_mem_oracle* or_mem_oracle_new(int kind, int ell, const uint64_t* r_point, int ell_addr, const uint64_t* r_addr,
                                 const uint64_t* init, int n_cols, const uint64_t* cols, const uint64_t* weights,
                                 uint64_t* claim_out);
void or_mem_oracle_free(or_mem_oracle* o);
int or_mem_oracle_num_rounds(const or_mem_oracle* o);
int or_mem_oracle_degree_bound(const or_mem_oracle* o);
void or_mem_oracle_evals(or_mem_oracle* o, const uint64_t* xs, int nx, uint64_t* ys);
void or_mem_oracle_fold(or_mem_oracle* o, const uint64_t* r);
void or_addr_lookup_weights(int ell, const uint64_t* r_cycle, int ell_addr, const uint64_t* has_lookup,
                            const uint64_t* addr_bits, const uint64_t* table, size_t table_len,
                            uint64_t* weights_out, uint64_t* claim_out);


/* Twist address-lane oracles (twist_oracle.rs:1259-1642); kind 0 read, 1 write. */
typedef struct or_twist_addr or_twist_addr;
or_twist_addr* or_twist_addr_new(int kind, int ell, const uint64_t* r_cycle, int ell_addr, size_t n_init,
                                 const uint64_t* init_addr, const uint64_t* init_val, const uint64_t* cols);
void or_twist_addr_free(or_twist_addr* o);
int or_twist_addr_num_rounds(const or_twist_addr* o);
void or_twist_addr_evals(or_twist_addr* o, const uint64_t* xs, int nx, uint64_t* ys);
void or_twist_addr_fold(or_twist_addr* o, const uint64_t* r);
void or_bus_openings(const int8_t* Z, int64_t m, int64_t bus_base, int64_t chunk, int n_cols, int64_t m_in,
                     const uint64_t* r, int ell, uint64_t* y_out, uint64_t* ysc_out);

#ifdef __cplusplus
}
#endif
#endif
