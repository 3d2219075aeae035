/*
 * neo_gpu.h -- C ABI of the B200 (sm_100a) Neo fold-step prover core.
 *
 * Plain C types only.  F_q = canonical uint64 < q (q = 2^64 - 2^32 + 1);
 * K = F_q[u]/(u^2 - 7) = two consecutive uint64 (re, im).  All buffers passed
 * to these functions are HOST buffers owned by the caller; they are copied to
 * and from the device inside the call.  Handles are opaque and freed by the
 * matching *_destroy.  Every function returns a status (NEO_OK = 0) and never
 * aborts; neo_gpu_last_error() gives the message of the last failure on a
 * context.  A context is bound to one device and one CUDA stream; calls on one
 * context must be serialized by the caller (one context per host thread).
 *
 * Each entry point cites the reference interface it replaces (path:line
 * relative to the reference project root).
 */
#ifndef NEO_GPU_H
#define NEO_GPU_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NEO_OK = 0,
    NEO_ERR_ARG = 1,        /* bad argument or shape (reference: panic / InvalidInput) */
    NEO_ERR_OOM = 2,        /* device allocation failed */
    NEO_ERR_INVARIANT = 3,  /* protocol invariant failed (reference: ProtocolError) */
    NEO_ERR_CUDA = 4,       /* CUDA runtime error */
    NEO_ERR_UNSUPPORTED = 5, /* parameter outside what the kernels implement */
    NEO_ERR_CANCELLED = 6    /* a batched request cancelled by neo_gpu_batch_cancel */
};

typedef struct neo_gpu_ctx neo_gpu_ctx;
typedef struct neo_gpu_ccs_oracle neo_gpu_ccs_oracle;

/* CCS structure (crates/neo-ccs/src/relations.rs:14-23).  Matrix j is the
 * identity sentinel when is_identity[j] != 0, otherwise CSC
 * (crates/neo-ccs/src/sparse.rs:19): column pointers col_ptr[j*(m+1) + c]
 * index into row_idx/vals starting at nnz_off[j].  f is a sparse polynomial
 * with n_terms terms: coefficient f_coeff[i], exponents f_exps[i*t + j]. */
typedef struct neo_ccs_desc {
    uint32_t n, m, t;
    const uint8_t* is_identity;
    const uint64_t* col_ptr;
    const uint64_t* nnz_off;
    const uint32_t* row_idx;
    const uint64_t* vals;
    uint32_t n_terms;
    const uint64_t* f_coeff;
    const uint32_t* f_exps;
} neo_ccs_desc;

/* ---- context -------------------------------------------------------- */
int neo_gpu_ctx_create(int device, neo_gpu_ctx** out);
int neo_gpu_ctx_destroy(neo_gpu_ctx* ctx);
const char* neo_gpu_last_error(const neo_gpu_ctx* ctx);
/* Bounded device wait (health check and test of the failure path): a kernel
 * polls a device flag at most spin_limit times (about 1 us apart, spin_limit
 * <= 2^20); set_flag != 0 sets the flag first.  NEO_OK when the flag was
 * seen; NEO_ERR_CUDA ("device wait timed out") when the wait ran out, with
 * the context left usable -- the same path the commitment kernel's bounded
 * mbarrier waits report through. */
int neo_gpu_wait_probe(neo_gpu_ctx* ctx, uint32_t set_flag, uint32_t spin_limit);
/* Number of kernels this context has launched so far (instrumentation). */
uint64_t neo_gpu_kernel_launches(const neo_gpu_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for event timing by callers. */
int neo_gpu_ctx_stream(const neo_gpu_ctx* ctx, void** stream);
/* Wait for the context's stream, then report and clear device-side errors: a
 * timed-out bounded wait (NEO_ERR_CUDA) or commitment digits that broke
 * NEO_COMMIT_SMALL_DIGITS (NEO_ERR_INVARIANT). */
int neo_gpu_synchronize(neo_gpu_ctx* ctx);

/* ---- Ajtai commitment (crates/neo-ajtai) ---------------------------- */
/* Upload public parameters M in R_q^{kappa x m}: coeffs[(i*m + j)*54 + s] is
 * coefficient s of M[i][j].  Replaces the PP registry load
 * (crates/neo-ajtai/src/s_module.rs:23-222, types.rs:7-16). */
int neo_gpu_pp_upload(neo_gpu_ctx* ctx, uint32_t kappa, uint64_t m, const uint64_t* coeffs);

/* Generate M on the device from a 32-byte ChaCha8 seed and register it like
 * neo_gpu_pp_upload.  mode NEO_PP_SETUP: setup(ChaCha8Rng::from_seed(seed),
 * 54, kappa, m) -- one stream, coefficient order [kappa][m][54]
 * (crates/neo-ajtai/src/commit.rs:133-157; FoldingSession::new_ajtai_seeded,
 * crates/neo-fold/src/session.rs:1938-1951).  mode NEO_PP_SETUP_PAR:
 * setup_par(ChaCha8Rng::from_seed(seed), 54, kappa, m) -- kappa row seeds,
 * per row one seed per chunk of min(m, 2^15).max(1024) columns
 * (commit.rs:159-225; seeded_pp_chunk_seeds, commit.rs:227-264;
 * FoldingSession::new_ajtai, session.rs:1915-1931).  Coefficients are drawn by
 * rejection (x < q) as sample_uniform_fq (commit.rs:21-30). */
#define NEO_PP_SETUP 0
#define NEO_PP_SETUP_PAR 1
int neo_gpu_pp_generate(neo_gpu_ctx* ctx, const uint8_t* seed32, uint32_t kappa, uint64_t m, int mode);

/* Copy words [first, first + count) of the registered PP of this m (layout
 * [kappa][m][54], word (i*m + j)*54 + s) back to the host. */
int neo_gpu_pp_download(neo_gpu_ctx* ctx, uint64_t m, uint64_t first, uint64_t count, uint64_t* out);

/* The sampler under neo_gpu_pp_generate: for each stream s (ChaCha8Rng seeded
 * with seeds[32*s .. 32*s+32]), the first counts[s] values x < bound of its
 * next_u64() sequence, concatenated into out.  bound = q is
 * sample_uniform_fq (crates/neo-ajtai/src/commit.rs:21-30); other bounds
 * exercise the rejection path. */
int neo_gpu_chacha8_sample(neo_gpu_ctx* ctx, const uint8_t* seeds, uint32_t n_streams, const uint64_t* counts,
                           uint64_t bound, uint64_t* out);

/* c = cf(M cf^{-1}(Z)) for n_vec digit matrices at once.
 * digits[(v*54 + r)*m + j] = Z_v[r][j] (row-major d x m, values in [-128,127]);
 * out[(v*kappa + i)*54 + r] = Commitment.data[i*54 + r] (column-major d x kappa,
 * crates/neo-ajtai/src/types.rs:17-50).  Replaces SModuleHomomorphism::commit
 * (crates/neo-ccs/src/traits.rs:8-14; crates/neo-ajtai/src/s_module.rs:335-377)
 * and commit_row_major (crates/neo-ajtai/src/commit.rs:376-402, 679-744). */
int neo_gpu_commit(neo_gpu_ctx* ctx, const int8_t* digits, uint32_t n_vec, uint64_t m, uint64_t* out);

/* neo_gpu_commit with DEVICE pointers (digits and out already in HBM); the
 * call is asynchronous on the context stream.  (neo_gpu_commit checks the
 * digits once and takes the faster small-digit tensor-core form when every
 * |digit| <= 63; this call, which never synchronizes, takes the form valid for
 * any int8 unless neo_gpu_commit_device_ex says the digits are small.) */
int neo_gpu_commit_device(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m, uint64_t* d_out);

/* neo_gpu_commit_device with flags.  NEO_COMMIT_SMALL_DIGITS: the caller
 * guarantees |digit| <= 63 (balanced base-b digits, b <= 64, as
 * decomp_b_row_major produces, crates/neo-ajtai/src/decomp.rs:118-158), so
 * the product is taken mod Phi_81 directly on the tensor cores, whose operand
 * entries are sums of two digits.  Digits outside the guarantee whose sums
 * leave int8 (the result would be wrong) are reported as NEO_ERR_INVARIANT by
 * the next call that checks the context's device error word
 * (neo_gpu_synchronize); otherwise the result is exact.
 * Asynchronous on the context stream. */
#define NEO_COMMIT_SMALL_DIGITS 1u
int neo_gpu_commit_device_ex(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m, uint64_t* d_out,
                             uint32_t flags);

/* Allocation-free commitment (no counterpart in the reference).  Same result
 * as neo_gpu_commit_device, for callers that cannot allocate device memory
 * when they commit: code running under CUDA stream capture, hosts whose
 * framework owns all device memory through its own pool, and latency-critical
 * provers that cannot afford the implicit synchronization of cudaMalloc /
 * cudaFree.  Inputs and outputs are DEVICE pointers owned by the caller; the
 * split-K scratch is a fixed 4 MiB device array inside the library (held by
 * every GPU that loads the library until exit).  n_vec * kappa * 81 must not
 * exceed 524288 (n_vec <= 404 for kappa = 16), else NEO_ERR_ARG.  The first
 * call on a device resolves the array's device address (cudaGetSymbolAddress):
 * make that first call before any stream capture.  All calls share the array,
 * so calls that overlap on the GPU (other streams or contexts) race.  The call
 * is asynchronous on the context stream and allocates nothing. */
int neo_gpu_commit_noalloc(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m, uint64_t* d_out);

/* Commitment mixers (CommitMixers, crates/neo-fold/src/shard.rs:146-153), host
 * buffers in and out.  Commitments are [kappa][54] F_q (Commitment::data,
 * column-major, crates/neo-ajtai/src/types.rs:15-22).
 * mix_rhos_commits: out = sum_i rho_i c_i with rhos[count][54][54] row-major
 * F_q matrices (the S-action of Pi_RLC, common.rs:398-430); cs[count][kappa][54].
 * combine_b_pows: out = sum_i b^i c_i (i from 0, the DEC parent check,
 * shard.rs:1120). */
int neo_gpu_mix_rhos_commits(neo_gpu_ctx* ctx, const uint64_t* rhos, const uint64_t* cs, uint32_t count,
                             uint32_t kappa, uint64_t* out);
int neo_gpu_combine_b_pows(neo_gpu_ctx* ctx, const uint64_t* cs, uint32_t count, uint32_t kappa, uint32_t b,
                           uint64_t* out);

/* Balanced base-2 decomposition z in F_q^m -> Z in {-1,0,1}^{54 x m}
 * row-major (crates/neo-ajtai/src/decomp.rs:118-158, DecompStyle::Balanced). */
int neo_gpu_decomp_b2(neo_gpu_ctx* ctx, const uint64_t* z, uint64_t m, int8_t* Z);

/* ---- Pi_RLC / Pi_DEC (crates/neo-reductions/src/common.rs) ---------- */
/* Z_mix = sum_i rot(a_i) Z_i, a_i = rho_coeffs[i*54 .. ] in {-2..2}
 * (common.rs:398-430 rot_from_coeffs; optimized_engine/common.rs:1221-1379).
 * Zs[(i*54 + r)*m + c]; Zmix[r*m + c] exact small integers. count == 1 is the
 * identity (common.rs:560-564). */
int neo_gpu_rlc_mix(neo_gpu_ctx* ctx, const int8_t* rho_coeffs, const int8_t* Zs, uint32_t count,
                    uint64_t m, int32_t* Zmix);

/* Balanced base-b split into k planes with nonzero flags
 * (common.rs:75-268 split_b_matrix_k_with_nonzero_flags).  Returns
 * NEO_ERR_INVARIANT when an entry needs more than k digits. */
int neo_gpu_split_b(neo_gpu_ctx* ctx, const int32_t* Zmix, uint64_t len, uint32_t k, uint32_t b,
                    int8_t* planes, uint8_t* nonzero);

/* y_j = Z (M_j^T chi_r) for every CCS matrix j, and y_scalars_j = sum_rho b^rho y_j[rho]
 * (common.rs:582-650 compute_y_from_Z_and_r).  Z: n_w digit matrices [n_w][54][m];
 * r: ell_n K points; y: [n_w][t][54] K; y_scalars: [n_w][t] K. */
int neo_gpu_me_y(neo_gpu_ctx* ctx, const neo_ccs_desc* ccs, const int8_t* Z, uint32_t n_w,
                 uint32_t ell_n, const uint64_t* r, uint32_t b, uint64_t* y, uint64_t* y_scalars);

/* ---- Pi_CCS sum-check oracle (RoundOracle) -------------------------- */
/* OptimizedOracle::new_with_sparse
 * (crates/neo-reductions/src/engines/optimized_engine/oracle.rs:1597-1639,
 * RowStreamState::build oracle.rs:82-414).  Z: [k][54][m] digits, MCS
 * witnesses first then ME witnesses; alpha, beta_a: ell_d K; beta_r: ell_n K;
 * gamma: 1 K; r_inputs: ell_n K or NULL.  Requires n == m == 2^ell_n and b == 2.
 * The oracle keeps its own device copy of Z and the CCS. */
int neo_gpu_ccs_oracle_create(neo_gpu_ctx* ctx, const neo_ccs_desc* ccs, const int8_t* Z, uint32_t k,
                              uint32_t b, const uint64_t* alpha, const uint64_t* beta_a,
                              const uint64_t* beta_r, const uint64_t* gamma, const uint64_t* r_inputs,
                              uint32_t ell_d, uint32_t ell_n, uint32_t d_sc, neo_gpu_ccs_oracle** out);
/* RoundOracle::evals_at (crates/neo-reductions/src/sumcheck.rs:17-34;
 * oracle.rs:2087-2093): ys[i] = p_round(xs[i]). */
int neo_gpu_ccs_oracle_evals(neo_gpu_ccs_oracle* o, const uint64_t* xs, uint32_t nx, uint64_t* ys);
/* RoundOracle::fold (oracle.rs:2095-2103). */
int neo_gpu_ccs_oracle_fold(neo_gpu_ccs_oracle* o, const uint64_t* r);
/* No counterpart in the reference (its rounds are driven one at a time by the
 * transcript): runs the next n row rounds back to back with caller-chosen
 * challenges chals[n] (host K), writing each round polynomial's d_sc + 1
 * coefficients (lowest first) to d_coeffs[n][d_sc + 1] (device K), with no
 * host synchronisation in between.  For fixed-challenge replays, benchmarks
 * and graph capture; the oracle is left after those n folds. */
int neo_gpu_ccs_oracle_row_rounds_device(neo_gpu_ccs_oracle* o, const uint64_t* chals, uint32_t n,
                                         uint64_t* d_coeffs);
uint32_t neo_gpu_ccs_oracle_num_rounds(const neo_gpu_ccs_oracle* o);
uint32_t neo_gpu_ccs_oracle_degree_bound(const neo_gpu_ccs_oracle* o);
/* build_me_outputs_from_ajtai_precomp (oracle.rs:1955-2072), after the
 * ell_n row rounds: y [k][t][54] K digits and y_scalars [k][t] K. */
int neo_gpu_ccs_oracle_me_outputs(neo_gpu_ccs_oracle* o, uint64_t* y, uint64_t* y_scalars);
int neo_gpu_ccs_oracle_destroy(neo_gpu_ccs_oracle* o);

/* Launch-shape autotuner of the Pi_CCS row rounds (no counterpart in the
 * reference, whose oracle is CPU code): per shape (ell_n, k) the library keeps
 * the NC-block thread count, the out-of-line threshold and the histogram block
 * size that ran the row-round sequence fastest.  neo_gpu_ccs_autotune times
 * every candidate on the caller's CCS and k ternary digit matrices
 * Z[k][54][m] (n == m == 2^ell_n) with `reps` timed runs each and records the
 * best; out3 = {nc_threads, compact_q, hist_items}.  Oracles created later for
 * that shape use it.  neo_gpu_tune_save / neo_gpu_tune_load write / read the
 * table as text lines "ccs <ell_n> <k> <nc_threads> <compact_q> <hist_items>";
 * neo_gpu_tune_get reads one entry (NEO_ERR_ARG when the shape is untuned). */
int neo_gpu_ccs_autotune(neo_gpu_ctx* ctx, const neo_ccs_desc* ccs, const int8_t* Z, uint32_t k, uint32_t reps,
                         uint64_t* out3);
int neo_gpu_tune_load(const char* path);
int neo_gpu_tune_save(const char* path);
int neo_gpu_tune_get(uint32_t ell_n, uint32_t k, uint64_t* out3);

/* ---- Twist / Shout time-lane oracles (RoundOracle) ------------------- */
/* The sparse-in-time oracles of crates/neo-memory/src/twist_oracle.rs, on
 * dense tables.  cols: n_cols K columns of 2^ell entries each (column-major,
 * K = two u64), in this order per kind:
 *   SHOUT_VALUE    [has_lookup, val]                    ShoutValueOracleSparse::new (twist_oracle.rs:203-241)
 *   SHOUT_ADAPTER  [has_lookup, addr_bits x ell_addr]   IndexAdapterOracleSparseTime::new_with_gate (:384-437)
 *   BITNESS        [cols...], weights[n_cols]           LazyWeightedBitnessOracleSparseTime::new_with_cycle (:515-542)
 *   TWIST_READ     [has_read, rv, ra_bits x ell_addr, has_write, inc_at_write_addr, wa_bits x ell_addr]
 *                                                       TwistReadCheckOracleSparseTime::new (:622-682)
 *   TWIST_WRITE    [has_write, wv, inc_at_write_addr, wa_bits x ell_addr]
 *                                                       TwistWriteCheckOracleSparseTime::new (:767-824)
 *   VAL_EVAL       [has_write, inc_at_write_addr, wa_bits x ell_addr]  (r_point = r_time)
 *                                                       TwistValEvalOracleSparseTime::new (:911-974)
 *   TOTAL_INC      [has_write, inc_at_write_addr, wa_bits x ell_addr]  (no r_point)
 *                                                       TwistTotalIncOracleSparseTime::new (:1054-1102)
 *   PRODUCT        [factors...]  (degree bound = n_cols) ProductRoundOracle::new (:50-71)
 * r_point: r_cycle (ell K) for the χ-weighted kinds, r_time for VAL_EVAL.
 * init_at_r_addr: 1 K (Twist read / write).  *claim: the sum over the time
 * hypercube (the constructors' claimed sums; for bitness / read / write the
 * value the caller's claimed sum must equal).  Status 1 on a column count
 * that does not match the kind, 5 for a degree bound above 31. */
enum { NEO_MEM_SHOUT_VALUE = 0, NEO_MEM_SHOUT_ADAPTER = 1, NEO_MEM_BITNESS = 2, NEO_MEM_TWIST_READ = 3,
       NEO_MEM_TWIST_WRITE = 4, NEO_MEM_VAL_EVAL = 5, NEO_MEM_TOTAL_INC = 6, NEO_MEM_PRODUCT = 7 };
typedef struct neo_gpu_mem_oracle neo_gpu_mem_oracle;
int neo_gpu_mem_oracle_create(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point,
                              uint32_t ell_addr, const uint64_t* r_addr, const uint64_t* init_at_r_addr,
                              uint32_t n_cols, const uint64_t* cols, const uint64_t* weights, uint64_t* claim,
                              neo_gpu_mem_oracle** out);
/* Same with the columns in device memory (d_cols); points stay host. */
int neo_gpu_mem_oracle_create_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point,
                                     uint32_t ell_addr, const uint64_t* r_addr, const uint64_t* init_at_r_addr,
                                     uint32_t n_cols, const uint64_t* d_cols, const uint64_t* weights,
                                     uint64_t* claim, neo_gpu_mem_oracle** out);
/* RoundOracle::evals_at: ys[i] = p_round(xs[i]); after the last round every
 * point gets the final product (the reference's len == 1 branch). */
int neo_gpu_mem_oracle_evals(neo_gpu_mem_oracle* o, const uint64_t* xs, uint32_t nx, uint64_t* ys);
/* RoundOracle::fold; ignored once no rounds remain. */
int neo_gpu_mem_oracle_fold(neo_gpu_mem_oracle* o, const uint64_t* r);
uint32_t neo_gpu_mem_oracle_num_rounds(const neo_gpu_mem_oracle* o);
uint32_t neo_gpu_mem_oracle_degree_bound(const neo_gpu_mem_oracle* o);
int neo_gpu_mem_oracle_destroy(neo_gpu_mem_oracle* o);
/* AddressLookupOracle::new (twist_oracle.rs:1671-1724): weights[2^ell_addr]
 * with w[addr(t)] += χ_{r_cycle}(t)·has_lookup(t) (addr from bit columns
 * equal to one) and claim = Σ_a table[a]·w[a]; the address rounds are then a
 * PRODUCT oracle over [table, weights].  addr_bits: ell_addr columns of 2^ell. */
int neo_gpu_addr_lookup_weights(neo_gpu_ctx* ctx, uint32_t ell, const uint64_t* r_cycle, uint32_t ell_addr,
                                const uint64_t* has_lookup, const uint64_t* addr_bits, const uint64_t* table,
                                uint64_t table_len, uint64_t* weights, uint64_t* claim);

/* ---- Twist address-lane oracles (RoundOracle, degree 2) ---------------- */
/* TwistReadCheckAddrOracleSparseTime::new (kind 0, twist_oracle.rs:1259-1367)
 * and TwistWriteCheckAddrOracleSparseTime::new (kind 1, :1468-1548).
 * cols (2^ell K rows each) as for NEO_MEM_TWIST_READ / NEO_MEM_TWIST_WRITE;
 * init: n_init (address, K value) pairs of the initial memory
 * (MemInit::Sparse; addresses < 2^ell_addr).  Claimed sum: zero.  The
 * rounds bind the ell_addr address bits, low bit first; after the last
 * round every point evaluates to the final sum (the value the time-lane
 * check at r_addr must start from). */
typedef struct neo_gpu_twist_addr neo_gpu_twist_addr;
int neo_gpu_twist_addr_create(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle, uint32_t ell_addr,
                              uint64_t n_init, const uint64_t* init_addr, const uint64_t* init_val,
                              const uint64_t* cols, neo_gpu_twist_addr** out);
/* Same with the columns in device memory. */
int neo_gpu_twist_addr_create_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle,
                                     uint32_t ell_addr, uint64_t n_init, const uint64_t* init_addr,
                                     const uint64_t* init_val, const uint64_t* d_cols, neo_gpu_twist_addr** out);
int neo_gpu_twist_addr_evals(neo_gpu_twist_addr* o, const uint64_t* xs, uint32_t nx, uint64_t* ys);
int neo_gpu_twist_addr_fold(neo_gpu_twist_addr* o, const uint64_t* r);
uint32_t neo_gpu_twist_addr_num_rounds(const neo_gpu_twist_addr* o);
uint32_t neo_gpu_twist_addr_degree_bound(const neo_gpu_twist_addr* o);
int neo_gpu_twist_addr_destroy(neo_gpu_twist_addr* o);

/* ---- shard prove loop (crates/neo-fold/src/shard.rs:1725-2283) ------- */
typedef struct neo_gpu_shard neo_gpu_shard;
/* A shard prover over one CCS (n == m == 2^ell_n, identity-first, t <= 4,
 * b = 2) with its own Poseidon2 transcript (new(app_label)), a device-resident
 * accumulator and k_rho DEC children per step.  PP for this m must already be
 * uploaded on ctx.  Computes the CCS matrix digest
 * (crates/neo-reductions/src/engines/utils.rs:214-321) once. */
int neo_gpu_shard_create(neo_gpu_ctx* ctx, const neo_ccs_desc* ccs, uint32_t m_in, uint32_t k_rho,
                         const char* app_label, neo_gpu_shard** out);
/* One Twist memory or Shout lookup instance on the shared CPU bus
 * (neo-memory MemInstance / LutInstance, bit addressing: ell_addr = d * ell;
 * k, d, n_side, ell are bound into the transcript as given). */
typedef struct {
    uint32_t ell_addr;
    uint64_t k, d, n_side, ell;
    const uint64_t* table;        /* Shout: table_len F_q entries (NULL for Twist) */
    uint64_t table_len;
    uint64_t n_init;              /* Twist: MemInit::Sparse (address, value) pairs; 0 = MemInit::Zero */
    const uint64_t* init_addr;
    const uint64_t* init_val;
} neo_mem_instance;
/* The instances of every fold step of a shard.  `steps` trace steps per fold
 * step occupy the tail of z: bus cell (col, j) at z[m - bus_cols*steps +
 * col*steps + j], time row m_in + j, columns ordered as in
 * build_bus_layout_for_instances (neo-memory/src/cpu/bus_layout.rs:91-190):
 * every Shout [addr_bits.., has_lookup, val], then every Twist [ra_bits..,
 * wa_bits.., has_read, has_write, wv, rv, inc]. */
typedef struct {
    uint64_t steps;
    uint32_t n_shout;
    const neo_mem_instance* shout;
    uint32_t n_twist;
    const neo_mem_instance* twist;
} neo_mem_desc;
/* A shard prover whose fold steps also prove the Route-A memory sidecar
 * (fold_shard_prove_impl with a shared CPU bus, crates/neo-fold/src/
 * shard.rs:1803-2283; memory_sidecar/memory.rs:86-1670): Shout / Twist
 * address pre-time sum-checks, the Route-A time claims batched with the CCS
 * rounds, bus openings on every ME claim, the Twist val-eval batch and the
 * val lane (RLC + DEC of the CPU ME claims at r_val).  Shout instances share
 * one ell_addr; ell_addr <= 24. */
int neo_gpu_shard_create_mem(neo_gpu_ctx* ctx, const neo_ccs_desc* ccs, uint32_t m_in, uint32_t k_rho,
                             const char* app_label, const neo_mem_desc* mem, neo_gpu_shard** out);
/* Number of val-lane DEC children emitted so far (the reference's
 * val_lane_obligations, shard.rs:2548-2991). */
int neo_gpu_shard_val_obligations(const neo_gpu_shard* sh, uint64_t* count);
/* Checkpoint / resume: the state a shard carries from one fold step to the
 * next (transcript position, step index, accumulator instances and their
 * digit planes, the val lane's previous witness and commitment, Twist
 * MemInits, the previous step's bus columns) as one byte string; buf == NULL
 * only sets *len to its size (NEO_ERR_ARG when cap < *len).  A checkpoint
 * restores into a shard created with the same CCS, m_in, k_rho and memory
 * description, in any context or process (NEO_ERR_ARG otherwise, the shard
 * unchanged); its next fold steps then equal the uninterrupted shard's bit
 * for bit.  A serving loop evicts a shard's device state this way.  No
 * counterpart in the reference, whose prover keeps this state in memory for
 * the whole shard (crates/neo-fold/src/shard.rs:1725-2283). */
int neo_gpu_shard_checkpoint(neo_gpu_shard* sh, uint8_t* buf, uint64_t cap, uint64_t* len);
int neo_gpu_shard_restore(neo_gpu_shard* sh, const uint8_t* buf, uint64_t len);
/* Replace the initial state of Twist instance mem_idx for the following fold
 * steps: the MemInit of the next step's MemInstance, which for a trace split
 * into chunks is the memory state at the end of the previous chunk
 * (mem_init_from_state_map, crates/neo-memory/src/mem_init.rs:65-90).
 * n_init = 0: MemInit::Zero; otherwise MemInit::Sparse in canonical form
 * (addresses strictly increasing and < 2^ell_addr, mem_init.rs:26-60), else
 * NEO_ERR_ARG.  The public init digest absorbed per step follows it. */
int neo_gpu_shard_set_twist_init(neo_gpu_shard* sh, uint32_t mem_idx, uint64_t n_init, const uint64_t* init_addr,
                                 const uint64_t* init_val);
/* One fold step on the main lane (no Twist/Shout): witness build
 * (decomp + MCS commit, crates/neo-fold/src/session.rs:977-978), Pi_CCS
 * (batched time rounds + Ajtai rounds), ME outputs, Pi_RLC, Pi_DEC
 * (shard.rs:1803-2180, 1170-1331).  z: the step witness (m values, host).
 * proof: canonical dump of the step proof, in order: the MCS commitment
 * (kappa*54), the initial sum T (K), [Shout address pre-time: claimed sums,
 * active mask, round polynomials, r_addr], [per Twist: address round
 * polynomials, r_addr, read / write finals], the batched time round
 * polynomials (per round, per claim), the Ajtai round polynomials, the final
 * running sum, the ME outputs' y (k x t x 54 K) and y_scalars (k x t K), [the
 * bus openings of every output (bus_cols x 54 K + bus_cols K)], [Twist
 * val-eval: claimed sums, round polynomials, r_val, CPU ME claims at r_val
 * (y and y_scalars of (t + bus_cols) rows)], the main lane (k rhos x 54, the
 * parent commitment, per DEC child its commitment, core y (t x 54 K) and bus
 * y (bus_cols x 54 K)), [the val lane, same layout]; K = two words (re, im).
 * Pass NULL to query *proof_len. */
int neo_gpu_shard_fold_step(neo_gpu_shard* sh, const uint64_t* z, uint64_t* proof, uint64_t proof_cap,
                            uint64_t* proof_len);
/* The last fold step's proof in the field order of the reference's StepProof
 * (crates/neo-fold/src/shard_proof_types.rs:45-131) -- fold {ccs_out,
 * ccs_proof, rlc_rhos (54 x 54 Mat<F>), rlc_parent, dec_children}, mem
 * {cpu_me_claims_val, shout_addr_pre, per-Twist address proofs, the Twist
 * val-eval batch}, batched_time {claimed_sums, degree_bounds, labels,
 * round_polys[claim][round]}, val_fold -- as a canonical word dump: every Vec
 * prefixed by its length, K = (re, im), F and integers one word, [u8; 32]
 * digests four little-endian words, byte strings a length then 8 bytes per
 * word, Option a 0 / 1 word then the value.  MeInstance = {c (d, kappa,
 * data), X (rows, cols, data), r, y (rows of 2^ell_d K), y_scalars, m_in,
 * fold_digest, c_step_coords, u_offset, u_len}.  out == NULL only sets *len.
 * The CCS proof part is {sumcheck_rounds (the Ajtai rounds), Some(sc_initial_sum),
 * sumcheck_challenges (r' || alpha'), alpha, beta_a, beta_r, gamma,
 * sumcheck_final, header_digest (empty), _extra (None)}; a lane mixing one
 * instance carries rho = I. */
int neo_gpu_shard_step_proof(neo_gpu_shard* sh, uint64_t* out, uint64_t cap, uint64_t* len);
/* Same step with the witness already resident in device memory (d_z). */
int neo_gpu_shard_fold_step_device(neo_gpu_shard* sh, const uint64_t* d_z, uint64_t* proof_len);

/* The memory events of one chunk of a VM trace, per step j < steps: Shout
 * instance i (in neo_mem_desc order) looked up key[j] with value val[j] when
 * has_lookup[j] = 1; Twist instance i read rv[j] at ra[j] (has_read[j] = 1) and
 * wrote wv[j] at wa[j] (has_write[j] = 1).  Flags are 0 or 1; addresses and
 * values of inactive ports are ignored. */
typedef struct neo_shout_events {
    const uint8_t* has_lookup;
    const uint64_t* key;
    const uint64_t* val;
} neo_shout_events;
typedef struct neo_twist_events {
    const uint8_t* has_read;
    const uint64_t* ra;
    const uint64_t* rv;
    const uint8_t* has_write;
    const uint64_t* wa;
    const uint64_t* wv;
} neo_twist_events;
typedef struct neo_trace_chunk {
    uint64_t steps;                 /* <= the shard's steps per fold step (and <= 16384) */
    const neo_shout_events* shout;  /* one per Shout instance */
    const neo_twist_events* twist;  /* one per Twist instance */
} neo_trace_chunk;
/* One fold step built from a trace chunk on the device (the witness build of
 * R1csCpu::build_ccs_chunks with the shared CPU bus,
 * crates/neo-memory/src/cpu/r1cs_adapter.rs:372-650): z = z_cpu (the CPU
 * witness, z_cpu_len <= the bus base words) padded with zeros, the bus tail
 * written from the events (address bits least-significant first, flags,
 * values; bus cell (col, j) at bus_base + col*steps + j,
 * crates/neo-memory/src/cpu/bus_layout.rs:59-81), and each Twist write's
 * increment inc = wv - (the value at wa before the write) from a memory
 * state the shard keeps in device memory across chunks; then the step
 * proceeds as neo_gpu_shard_fold_step.  The step's Twist MemInit is that
 * state at the chunk's start (mem_init_from_state_map,
 * crates/neo-memory/src/mem_init.rs:65-90): after a successful step the
 * shard sets the next step's MemInit from it, so no
 * neo_gpu_shard_set_twist_init is needed between trace steps (one given
 * replaces the state).  An address >= 2^ell_addr, a flag other than 0 / 1 or
 * too many steps is NEO_ERR_ARG. */
int neo_gpu_shard_fold_step_trace(neo_gpu_shard* sh, const uint64_t* z_cpu, uint64_t z_cpu_len,
                                  const neo_trace_chunk* trace, uint64_t* proof, uint64_t proof_cap,
                                  uint64_t* proof_len);
/* Transcript sponge state (8 words) and CCS matrix digest (4 words). */
int neo_gpu_shard_transcript_state(const neo_gpu_shard* sh, uint64_t* st8);
int neo_gpu_shard_ccs_digest(const neo_gpu_shard* sh, uint64_t* d4);
/* Host milliseconds of the last step: [0] total, [1] witness decomp+commit,
 * [2] header/ME binding + challenges, [3] Pi_CCS table build, [4] memory
 * address pre-time + batched time rounds, [5] Ajtai rounds, [6] ME outputs,
 * [7] val-eval batch + main-lane Pi_RLC/Pi_DEC, [8] val lane; [9] transcript
 * permutations of the step; [10] memory-sidecar share of [4] and [7]. */
int neo_gpu_shard_step_stats(const neo_gpu_shard* sh, double* out, uint32_t n);
int neo_gpu_shard_destroy(neo_gpu_shard* sh);

/* ---- batched / served proving of many shards --------------------------- */
/* No single reference function: the reference proves shards one at a time
 * (crates/neo-fold/src/shard.rs:2285 fold_shard_prove).  A batch owns
 * n_workers host threads, each with its own context (CUDA stream) on `device`.
 * Submitted shard-prove requests (CCS + witness + number of fold steps) wait
 * in one FIFO queue; an idle worker starts the head request once its device
 * footprint fits (free HBM when the engine was last idle, minus the running
 * requests' footprints and the reserve) and proves it to completion.
 * Destroying the batch lets running requests finish; queued ones never start.
 * PP for every m used must be uploaded first (any context on the device). */
typedef struct neo_gpu_batch neo_gpu_batch;
int neo_gpu_batch_create(int device, uint32_t n_workers, neo_gpu_batch** out);
/* Device bytes kept free when admitting requests (default 2 GiB). */
int neo_gpu_batch_set_reserve(neo_gpu_batch* b, uint64_t bytes);
/* Inputs are copied; z has ccs->m words.  *job_id identifies the request. */
int neo_gpu_batch_submit(neo_gpu_batch* b, const neo_ccs_desc* ccs, const uint64_t* z, uint32_t n_steps,
                         uint32_t m_in, uint32_t k_rho, const char* app_label, uint64_t* job_id);
/* A request whose shard also proves the shared-CPU-bus memory sidecar
 * (mem as for neo_gpu_shard_create_mem; copied). */
int neo_gpu_batch_submit_mem(neo_gpu_batch* b, const neo_ccs_desc* ccs, const neo_mem_desc* mem, const uint64_t* z,
                             uint32_t n_steps, uint32_t m_in, uint32_t k_rho, const char* app_label,
                             uint64_t* job_id);
/* A request whose fold steps prove consecutive chunks of one trace: zs holds
 * n_steps witnesses of ccs->m words (step s proves zs[s*m ..]) and inits the
 * MemInit of every Twist instance before each step, row-major
 * [n_steps][mem->n_twist] (row 0 unused: the instances' own init; NULL: keep
 * them) -- what neo_gpu_shard_set_twist_init does between the steps of one
 * shard.  mem may have no instances (then inits is ignored). */
typedef struct {
    uint64_t n_init;        /* 0: MemInit::Zero */
    const uint64_t* addr;   /* strictly increasing, < 2^ell_addr */
    const uint64_t* val;
} neo_mem_init;
int neo_gpu_batch_submit_chunks(neo_gpu_batch* b, const neo_ccs_desc* ccs, const neo_mem_desc* mem,
                                const uint64_t* zs, const neo_mem_init* inits, uint32_t n_steps, uint32_t m_in,
                                uint32_t k_rho, const char* app_label, uint64_t* job_id);
/* Waits until every submitted request has finished (NEO_ERR_CUDA on timeout). */
int neo_gpu_batch_wait_all(neo_gpu_batch* b, double timeout_ms);
/* times3 = {submit->done ms, submit->admit ms, submit time since creation ms};
 * tr_state8 = final transcript state; status 1 = done, 0 = running, < 0 = -error. */
int neo_gpu_batch_job_info(neo_gpu_batch* b, uint64_t job_id, double* times3, uint64_t* tr_state8, int* status);
/* The error message of a failed request (empty while it runs or after it
 * succeeded), NUL-terminated and truncated to cap bytes. */
int neo_gpu_batch_job_error(neo_gpu_batch* b, uint64_t job_id, char* buf, uint64_t cap);
/* Cancels a request: a queued one never starts, a running one stops before
 * its next fold step (its device state is released); both finish with status
 * -NEO_ERR_CANCELLED.  A finished request is left as it is. */
int neo_gpu_batch_cancel(neo_gpu_batch* b, uint64_t job_id);
uint64_t neo_gpu_batch_kernel_launches(const neo_gpu_batch* b);
int neo_gpu_batch_destroy(neo_gpu_batch* b);

/* ---- Fiat-Shamir transcript (host only, no GPU needed) --------------- */
/* Poseidon2Transcript (crates/neo-transcript/src/poseidon2.rs:10-310):
 * width-8 overwrite sponge, rate 4, one field element per label byte. */
typedef struct neo_transcript neo_transcript;
int neo_transcript_new(const char* app_label, neo_transcript** out);
int neo_transcript_append_message(neo_transcript* t, const char* label, const uint8_t* msg, size_t len);
int neo_transcript_append_fields(neo_transcript* t, const char* label, const uint64_t* fs, size_t n);
int neo_transcript_append_u64s(neo_transcript* t, const char* label, const uint64_t* us, size_t n);
int neo_transcript_challenge_field(neo_transcript* t, const char* label, uint64_t* out);
int neo_transcript_challenge_fields(neo_transcript* t, const char* label, size_t n, uint64_t* out);
int neo_transcript_digest32(neo_transcript* t, uint8_t* out32);
int neo_transcript_state(const neo_transcript* t, uint64_t* st8);
int neo_transcript_destroy(neo_transcript* t);
/* digest_ccs_matrices (crates/neo-reductions/src/engines/utils.rs:214-321). */
int neo_ccs_digest(const neo_ccs_desc* ccs, uint64_t* out4);

#ifdef __cplusplus
}
#endif
#endif
