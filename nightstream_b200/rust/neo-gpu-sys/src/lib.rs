//! Raw FFI bindings to libneo_gpu.so, one declaration per entry point of
//! include/neo_gpu.h (same names, argument order and meaning).  Every
//! function returns a status (0 = ok; NEO_ERR_* otherwise, the message from
//! `neo_gpu_last_error`); field elements are canonical u64 < q, K elements two
//! consecutive u64 (re, im).  Safe wrappers and the reference trait impls live
//! in the `neo-gpu` crate beside this one.
#![allow(non_camel_case_types, non_snake_case, clippy::missing_safety_doc)]

use core::ffi::{c_char, c_int, c_void};

pub const NEO_OK: c_int = 0;
pub const NEO_ERR_ARG: c_int = 1;
pub const NEO_ERR_OOM: c_int = 2;
pub const NEO_ERR_INVARIANT: c_int = 3;
pub const NEO_ERR_CUDA: c_int = 4;
pub const NEO_ERR_UNSUPPORTED: c_int = 5;
pub const NEO_ERR_CANCELLED: c_int = 6;
pub const NEO_COMMIT_SMALL_DIGITS: u32 = 1;

/// Memory-oracle kinds (include/neo_gpu.h, NEO_MEM_*).
pub const NEO_MEM_SHOUT_VALUE: c_int = 0;
pub const NEO_MEM_SHOUT_ADAPTER: c_int = 1;
pub const NEO_MEM_BITNESS: c_int = 2;
pub const NEO_MEM_TWIST_READ: c_int = 3;
pub const NEO_MEM_TWIST_WRITE: c_int = 4;
pub const NEO_MEM_VAL_EVAL: c_int = 5;
pub const NEO_MEM_TOTAL_INC: c_int = 6;
pub const NEO_MEM_PRODUCT: c_int = 7;

macro_rules! opaque {
    ($($name:ident),*) => { $( #[repr(C)] pub struct $name { _private: [u8; 0] } )* };
}
opaque!(neo_gpu_ctx, neo_gpu_ccs_oracle, neo_gpu_mem_oracle, neo_gpu_twist_addr, neo_gpu_shard, neo_gpu_batch,
        neo_transcript);

/// CCS structure: matrix j is the identity when is_identity[j] != 0, else CSC
/// with column pointers col_ptr[j*(m+1) + c] into row_idx / vals from
/// nnz_off[j]; f has n_terms terms (f_coeff[i], exponents f_exps[i*t + j]).
#[repr(C)]
#[derive(Clone, Copy)]
pub struct neo_ccs_desc {
    pub n: u32,
    pub m: u32,
    pub t: u32,
    pub is_identity: *const u8,
    pub col_ptr: *const u64,
    pub nnz_off: *const u64,
    pub row_idx: *const u32,
    pub vals: *const u64,
    pub n_terms: u32,
    pub f_coeff: *const u64,
    pub f_exps: *const u32,
}

/// One Twist (read/write memory) or Shout (lookup table) instance on the shared CPU bus.
#[repr(C)]
#[derive(Clone, Copy)]
pub struct neo_mem_instance {
    pub ell_addr: u32,
    pub k: u64,
    pub d: u64,
    pub n_side: u64,
    pub ell: u64,
    pub table: *const u64,
    pub table_len: u64,
    pub n_init: u64,
    pub init_addr: *const u64,
    pub init_val: *const u64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct neo_mem_desc {
    pub steps: u64,
    pub n_shout: u32,
    pub shout: *const neo_mem_instance,
    pub n_twist: u32,
    pub twist: *const neo_mem_instance,
}

/// One Shout instance's events of a trace chunk (include/neo_gpu.h).
#[repr(C)]
#[derive(Clone, Copy)]
pub struct neo_shout_events {
    pub has_lookup: *const u8,
    pub key: *const u64,
    pub val: *const u64,
}

/// One Twist instance's events of a trace chunk.
#[repr(C)]
#[derive(Clone, Copy)]
pub struct neo_twist_events {
    pub has_read: *const u8,
    pub ra: *const u64,
    pub rv: *const u64,
    pub has_write: *const u8,
    pub wa: *const u64,
    pub wv: *const u64,
}

/// The memory events of one trace chunk (neo_gpu_shard_fold_step_trace).
#[repr(C)]
#[derive(Clone, Copy)]
pub struct neo_trace_chunk {
    pub steps: u64,
    pub shout: *const neo_shout_events,
    pub twist: *const neo_twist_events,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct neo_mem_init {
    pub n_init: u64,
    pub addr: *const u64,
    pub val: *const u64,
}

extern "C" {
    pub fn neo_gpu_ctx_create(device: c_int, out: *mut *mut neo_gpu_ctx) -> c_int;
    pub fn neo_gpu_ctx_destroy(ctx: *mut neo_gpu_ctx) -> c_int;
    pub fn neo_gpu_last_error(ctx: *const neo_gpu_ctx) -> *const c_char;
    pub fn neo_gpu_wait_probe(ctx: *mut neo_gpu_ctx, set_flag: u32, spin_limit: u32) -> c_int;
    pub fn neo_gpu_ctx_stream(ctx: *const neo_gpu_ctx, stream: *mut *mut c_void) -> c_int;
    pub fn neo_gpu_synchronize(ctx: *mut neo_gpu_ctx) -> c_int;
    pub fn neo_gpu_pp_upload(ctx: *mut neo_gpu_ctx, kappa: u32, m: u64, coeffs: *const u64) -> c_int;
    pub fn neo_gpu_pp_generate(ctx: *mut neo_gpu_ctx, seed32: *const u8, kappa: u32, m: u64, mode: c_int) -> c_int;
    pub fn neo_gpu_pp_download(ctx: *mut neo_gpu_ctx, m: u64, first: u64, count: u64, out: *mut u64) -> c_int;
    pub fn neo_gpu_chacha8_sample(ctx: *mut neo_gpu_ctx, seeds: *const u8, n_streams: u32, counts: *const u64, bound: u64, out: *mut u64) -> c_int;
    pub fn neo_gpu_commit(ctx: *mut neo_gpu_ctx, digits: *const i8, n_vec: u32, m: u64, out: *mut u64) -> c_int;
    pub fn neo_gpu_commit_device(ctx: *mut neo_gpu_ctx, d_digits: *const i8, n_vec: u32, m: u64, d_out: *mut u64) -> c_int;
    pub fn neo_gpu_commit_device_ex(ctx: *mut neo_gpu_ctx, d_digits: *const i8, n_vec: u32, m: u64, d_out: *mut u64, flags: u32) -> c_int;
    pub fn neo_gpu_commit_noalloc(ctx: *mut neo_gpu_ctx, d_digits: *const i8, n_vec: u32, m: u64, d_out: *mut u64) -> c_int;
    pub fn neo_gpu_mix_rhos_commits(ctx: *mut neo_gpu_ctx, rhos: *const u64, cs: *const u64, count: u32, kappa: u32, out: *mut u64) -> c_int;
    pub fn neo_gpu_combine_b_pows(ctx: *mut neo_gpu_ctx, cs: *const u64, count: u32, kappa: u32, b: u32, out: *mut u64) -> c_int;
    pub fn neo_gpu_decomp_b2(ctx: *mut neo_gpu_ctx, z: *const u64, m: u64, Z: *mut i8) -> c_int;
    pub fn neo_gpu_rlc_mix(ctx: *mut neo_gpu_ctx, rho_coeffs: *const i8, Zs: *const i8, count: u32, m: u64, Zmix: *mut i32) -> c_int;
    pub fn neo_gpu_split_b(ctx: *mut neo_gpu_ctx, Zmix: *const i32, len: u64, k: u32, b: u32, planes: *mut i8, nonzero: *mut u8) -> c_int;
    pub fn neo_gpu_me_y(ctx: *mut neo_gpu_ctx, ccs: *const neo_ccs_desc, Z: *const i8, n_w: u32, ell_n: u32, r: *const u64, b: u32, y: *mut u64, y_scalars: *mut u64) -> c_int;
    pub fn neo_gpu_ccs_oracle_create(ctx: *mut neo_gpu_ctx, ccs: *const neo_ccs_desc, Z: *const i8, k: u32, b: u32, alpha: *const u64, beta_a: *const u64, beta_r: *const u64, gamma: *const u64, r_inputs: *const u64, ell_d: u32, ell_n: u32, d_sc: u32, out: *mut *mut neo_gpu_ccs_oracle) -> c_int;
    pub fn neo_gpu_ccs_oracle_evals(o: *mut neo_gpu_ccs_oracle, xs: *const u64, nx: u32, ys: *mut u64) -> c_int;
    pub fn neo_gpu_ccs_oracle_fold(o: *mut neo_gpu_ccs_oracle, r: *const u64) -> c_int;
    pub fn neo_gpu_ccs_oracle_row_rounds_device(o: *mut neo_gpu_ccs_oracle, chals: *const u64, n: u32, d_coeffs: *mut u64) -> c_int;
    pub fn neo_gpu_ccs_oracle_num_rounds(o: *const neo_gpu_ccs_oracle) -> u32;
    pub fn neo_gpu_ccs_oracle_degree_bound(o: *const neo_gpu_ccs_oracle) -> u32;
    pub fn neo_gpu_ccs_oracle_me_outputs(o: *mut neo_gpu_ccs_oracle, y: *mut u64, y_scalars: *mut u64) -> c_int;
    pub fn neo_gpu_ccs_oracle_destroy(o: *mut neo_gpu_ccs_oracle) -> c_int;
    pub fn neo_gpu_ccs_autotune(ctx: *mut neo_gpu_ctx, ccs: *const neo_ccs_desc, Z: *const i8, k: u32, reps: u32, out3: *mut u64) -> c_int;
    pub fn neo_gpu_tune_load(path: *const c_char) -> c_int;
    pub fn neo_gpu_tune_save(path: *const c_char) -> c_int;
    pub fn neo_gpu_tune_get(ell_n: u32, k: u32, out3: *mut u64) -> c_int;
    pub fn neo_gpu_mem_oracle_create(ctx: *mut neo_gpu_ctx, kind: c_int, ell: u32, r_point: *const u64, ell_addr: u32, r_addr: *const u64, init_at_r_addr: *const u64, n_cols: u32, cols: *const u64, weights: *const u64, claim: *mut u64, out: *mut *mut neo_gpu_mem_oracle) -> c_int;
    pub fn neo_gpu_mem_oracle_create_device(ctx: *mut neo_gpu_ctx, kind: c_int, ell: u32, r_point: *const u64, ell_addr: u32, r_addr: *const u64, init_at_r_addr: *const u64, n_cols: u32, d_cols: *const u64, weights: *const u64, claim: *mut u64, out: *mut *mut neo_gpu_mem_oracle) -> c_int;
    pub fn neo_gpu_mem_oracle_evals(o: *mut neo_gpu_mem_oracle, xs: *const u64, nx: u32, ys: *mut u64) -> c_int;
    pub fn neo_gpu_mem_oracle_fold(o: *mut neo_gpu_mem_oracle, r: *const u64) -> c_int;
    pub fn neo_gpu_mem_oracle_num_rounds(o: *const neo_gpu_mem_oracle) -> u32;
    pub fn neo_gpu_mem_oracle_degree_bound(o: *const neo_gpu_mem_oracle) -> u32;
    pub fn neo_gpu_mem_oracle_destroy(o: *mut neo_gpu_mem_oracle) -> c_int;
    pub fn neo_gpu_addr_lookup_weights(ctx: *mut neo_gpu_ctx, ell: u32, r_cycle: *const u64, ell_addr: u32, has_lookup: *const u64, addr_bits: *const u64, table: *const u64, table_len: u64, weights: *mut u64, claim: *mut u64) -> c_int;
    pub fn neo_gpu_twist_addr_create(ctx: *mut neo_gpu_ctx, kind: c_int, ell: u32, r_cycle: *const u64, ell_addr: u32, n_init: u64, init_addr: *const u64, init_val: *const u64, cols: *const u64, out: *mut *mut neo_gpu_twist_addr) -> c_int;
    pub fn neo_gpu_twist_addr_create_device(ctx: *mut neo_gpu_ctx, kind: c_int, ell: u32, r_cycle: *const u64, ell_addr: u32, n_init: u64, init_addr: *const u64, init_val: *const u64, d_cols: *const u64, out: *mut *mut neo_gpu_twist_addr) -> c_int;
    pub fn neo_gpu_twist_addr_evals(o: *mut neo_gpu_twist_addr, xs: *const u64, nx: u32, ys: *mut u64) -> c_int;
    pub fn neo_gpu_twist_addr_fold(o: *mut neo_gpu_twist_addr, r: *const u64) -> c_int;
    pub fn neo_gpu_twist_addr_num_rounds(o: *const neo_gpu_twist_addr) -> u32;
    pub fn neo_gpu_twist_addr_degree_bound(o: *const neo_gpu_twist_addr) -> u32;
    pub fn neo_gpu_twist_addr_destroy(o: *mut neo_gpu_twist_addr) -> c_int;
    pub fn neo_gpu_shard_create(ctx: *mut neo_gpu_ctx, ccs: *const neo_ccs_desc, m_in: u32, k_rho: u32, app_label: *const c_char, out: *mut *mut neo_gpu_shard) -> c_int;
    pub fn neo_gpu_shard_create_mem(ctx: *mut neo_gpu_ctx, ccs: *const neo_ccs_desc, m_in: u32, k_rho: u32, app_label: *const c_char, mem: *const neo_mem_desc, out: *mut *mut neo_gpu_shard) -> c_int;
    pub fn neo_gpu_shard_val_obligations(sh: *const neo_gpu_shard, count: *mut u64) -> c_int;
    pub fn neo_gpu_shard_checkpoint(sh: *mut neo_gpu_shard, buf: *mut u8, cap: u64, len: *mut u64) -> c_int;
    pub fn neo_gpu_shard_restore(sh: *mut neo_gpu_shard, buf: *const u8, len: u64) -> c_int;
    pub fn neo_gpu_shard_set_twist_init(sh: *mut neo_gpu_shard, mem_idx: u32, n_init: u64, init_addr: *const u64, init_val: *const u64) -> c_int;
    pub fn neo_gpu_shard_fold_step(sh: *mut neo_gpu_shard, z: *const u64, proof: *mut u64, proof_cap: u64, proof_len: *mut u64) -> c_int;
    pub fn neo_gpu_shard_step_proof(sh: *mut neo_gpu_shard, out: *mut u64, cap: u64, len: *mut u64) -> c_int;
    pub fn neo_gpu_shard_fold_step_device(sh: *mut neo_gpu_shard, d_z: *const u64, proof_len: *mut u64) -> c_int;
    pub fn neo_gpu_shard_fold_step_trace(sh: *mut neo_gpu_shard, z_cpu: *const u64, z_cpu_len: u64, trace: *const neo_trace_chunk, proof: *mut u64, proof_cap: u64, proof_len: *mut u64) -> c_int;
    pub fn neo_gpu_shard_transcript_state(sh: *const neo_gpu_shard, st8: *mut u64) -> c_int;
    pub fn neo_gpu_shard_ccs_digest(sh: *const neo_gpu_shard, d4: *mut u64) -> c_int;
    pub fn neo_gpu_shard_step_stats(sh: *const neo_gpu_shard, out: *mut f64, n: u32) -> c_int;
    pub fn neo_gpu_shard_destroy(sh: *mut neo_gpu_shard) -> c_int;
    pub fn neo_gpu_batch_create(device: c_int, n_workers: u32, out: *mut *mut neo_gpu_batch) -> c_int;
    pub fn neo_gpu_batch_set_reserve(b: *mut neo_gpu_batch, bytes: u64) -> c_int;
    pub fn neo_gpu_batch_submit(b: *mut neo_gpu_batch, ccs: *const neo_ccs_desc, z: *const u64, n_steps: u32, m_in: u32, k_rho: u32, app_label: *const c_char, job_id: *mut u64) -> c_int;
    pub fn neo_gpu_batch_submit_mem(b: *mut neo_gpu_batch, ccs: *const neo_ccs_desc, mem: *const neo_mem_desc, z: *const u64, n_steps: u32, m_in: u32, k_rho: u32, app_label: *const c_char, job_id: *mut u64) -> c_int;
    pub fn neo_gpu_batch_submit_chunks(b: *mut neo_gpu_batch, ccs: *const neo_ccs_desc, mem: *const neo_mem_desc, zs: *const u64, inits: *const neo_mem_init, n_steps: u32, m_in: u32, k_rho: u32, app_label: *const c_char, job_id: *mut u64) -> c_int;
    pub fn neo_gpu_batch_wait_all(b: *mut neo_gpu_batch, timeout_ms: f64) -> c_int;
    pub fn neo_gpu_batch_job_info(b: *mut neo_gpu_batch, job_id: u64, times3: *mut f64, tr_state8: *mut u64, status: *mut c_int) -> c_int;
    pub fn neo_gpu_batch_job_error(b: *mut neo_gpu_batch, job_id: u64, buf: *mut c_char, cap: u64) -> c_int;
    pub fn neo_gpu_batch_cancel(b: *mut neo_gpu_batch, job_id: u64) -> c_int;
    pub fn neo_gpu_batch_destroy(b: *mut neo_gpu_batch) -> c_int;
    pub fn neo_transcript_new(app_label: *const c_char, out: *mut *mut neo_transcript) -> c_int;
    pub fn neo_transcript_append_message(t: *mut neo_transcript, label: *const c_char, msg: *const u8, len: usize) -> c_int;
    pub fn neo_transcript_append_fields(t: *mut neo_transcript, label: *const c_char, fs: *const u64, n: usize) -> c_int;
    pub fn neo_transcript_append_u64s(t: *mut neo_transcript, label: *const c_char, us: *const u64, n: usize) -> c_int;
    pub fn neo_transcript_challenge_field(t: *mut neo_transcript, label: *const c_char, out: *mut u64) -> c_int;
    pub fn neo_transcript_challenge_fields(t: *mut neo_transcript, label: *const c_char, n: usize, out: *mut u64) -> c_int;
    pub fn neo_transcript_digest32(t: *mut neo_transcript, out32: *mut u8) -> c_int;
    pub fn neo_transcript_state(t: *const neo_transcript, st8: *mut u64) -> c_int;
    pub fn neo_transcript_destroy(t: *mut neo_transcript) -> c_int;
    pub fn neo_ccs_digest(ccs: *const neo_ccs_desc, out4: *mut u64) -> c_int;
}
