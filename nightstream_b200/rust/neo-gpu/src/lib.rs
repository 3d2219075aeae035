//! The GPU prover core beneath the reference's trait surfaces.
//!
//! * [`GpuCcsOracle`] implements `neo_reductions::sumcheck::RoundOracle`
//!   (crates/neo-reductions/src/sumcheck.rs:17-34) for Pi_CCS;
//!   [`GpuMemOracle`] and [`GpuTwistAddr`] do the same for the Twist / Shout
//!   time-lane and address-lane oracles (crates/neo-memory/src/twist_oracle.rs).
//! * [`GpuAjtai`] implements `neo_ccs::traits::SModuleHomomorphism<F, Commitment>`
//!   (crates/neo-ccs/src/traits.rs:8-14) with the tensor-core commitment.
//! * [`Context::mix_rhos_commits`] / [`Context::combine_b_pows`] have the
//!   signatures of the `CommitMixers` closures (crates/neo-fold/src/shard.rs:146-153).
//!
//! The reference's trait methods are infallible and panic on shape errors; the
//! impls here do the same with the library's error message.  Field elements
//! cross the boundary as canonical u64, K elements as (re, im).
use core::ffi::{c_char, CStr};
use neo_ajtai::Commitment;
use neo_ccs::relations::CcsStructure;
use neo_ccs::sparse::CcsMatrix;
use neo_ccs::traits::SModuleHomomorphism;
use neo_ccs::Mat;
use neo_gpu_sys as sys;
use neo_math::{from_complex, KExtensions, F, K};
use neo_reductions::sumcheck::RoundOracle;
use p3_field::{PrimeCharacteristicRing, PrimeField64};

/// A failed library call: the status code (sys::NEO_ERR_*) and its message.
#[derive(Debug, Clone)]
pub struct Error {
    pub code: i32,
    pub msg: String,
}

impl core::fmt::Display for Error {
    fn fmt(&self, f: &mut core::fmt::Formatter<'_>) -> core::fmt::Result {
        write!(f, "neo_gpu error {}: {}", self.code, self.msg)
    }
}

pub type Result<T> = core::result::Result<T, Error>;

fn k_words(k: &K) -> [u64; 2] {
    [k.real().as_canonical_u64(), k.imag().as_canonical_u64()]
}

fn k_from(w: &[u64]) -> K {
    from_complex(F::from_u64(w[0]), F::from_u64(w[1]))
}

fn flat_k(ks: &[K]) -> Vec<u64> {
    ks.iter().flat_map(k_words).collect()
}

/// A balanced digit matrix (d x m, row-major) as int8; panics on an entry
/// outside [-127, 127] (the GPU commitment and oracles take digit planes).
fn digits_i8(z: &Mat<F>) -> Vec<i8> {
    const Q: u64 = 0xFFFF_FFFF_0000_0001;
    z.as_slice()
        .iter()
        .map(|x| {
            let u = x.as_canonical_u64();
            if u <= 127 {
                u as i8
            } else if u >= Q - 127 {
                -((Q - u) as i64) as i8
            } else {
                panic!("neo-gpu: matrix entry {u} is not a small balanced digit")
            }
        })
        .collect()
}

/// One GPU context (its own CUDA stream).  A context is used by one thread at a time.
pub struct Context {
    raw: *mut sys::neo_gpu_ctx,
}

unsafe impl Send for Context {}

impl Context {
    pub fn new(device: i32) -> Result<Self> {
        let mut raw = core::ptr::null_mut();
        let rc = unsafe { sys::neo_gpu_ctx_create(device, &mut raw) };
        if rc != 0 {
            return Err(Error { code: rc, msg: "neo_gpu_ctx_create".into() });
        }
        Ok(Self { raw })
    }

    pub fn raw(&self) -> *mut sys::neo_gpu_ctx {
        self.raw
    }

    fn check(&self, rc: i32) -> Result<()> {
        if rc == 0 {
            return Ok(());
        }
        let msg = unsafe {
            let p: *const c_char = sys::neo_gpu_last_error(self.raw);
            if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
        };
        Err(Error { code: rc, msg })
    }

    /// setup / setup_par (mode 0 / 1) from ChaCha8Rng::from_seed(seed) on the
    /// device, registered for commitments of width m (crates/neo-ajtai/src/commit.rs:133-264).
    pub fn pp_generate(&self, seed: &[u8; 32], kappa: u32, m: u64, par: bool) -> Result<()> {
        self.check(unsafe { sys::neo_gpu_pp_generate(self.raw, seed.as_ptr(), kappa, m, par as i32) })
    }

    /// Registers a PP made by the caller: coeffs [kappa][m][54] canonical.
    pub fn pp_upload(&self, kappa: u32, m: u64, coeffs: &[u64]) -> Result<()> {
        assert_eq!(coeffs.len() as u64, kappa as u64 * m * 54, "pp_upload: shape");
        self.check(unsafe { sys::neo_gpu_pp_upload(self.raw, kappa, m, coeffs.as_ptr()) })
    }

    /// Commitments of n_vec digit matrices [n_vec][54][m] -> [n_vec][kappa][54].
    pub fn commit_digits(&self, digits: &[i8], n_vec: u32, m: u64, kappa: u32) -> Result<Vec<u64>> {
        assert_eq!(digits.len() as u64, n_vec as u64 * 54 * m, "commit: shape");
        let mut out = vec![0u64; (n_vec * kappa * 54) as usize];
        self.check(unsafe { sys::neo_gpu_commit(self.raw, digits.as_ptr(), n_vec, m, out.as_mut_ptr()) })?;
        Ok(out)
    }

    /// CommitMixers::mix_rhos_commits: sum_i rho_i c_i.
    pub fn mix_rhos_commits(&self, rhos: &[Mat<F>], cs: &[Commitment]) -> Commitment {
        assert_eq!(rhos.len(), cs.len(), "mix_rhos_commits: |rhos| != |cs|");
        assert!(!cs.is_empty(), "mix_rhos_commits: no commitments");
        let kappa = cs[0].kappa;
        let mut r = Vec::with_capacity(rhos.len() * 54 * 54);
        for m in rhos {
            assert!(m.rows() == 54 && m.cols() == 54, "mix_rhos_commits: rho must be 54 x 54");
            r.extend(m.as_slice().iter().map(|x| x.as_canonical_u64()));
        }
        let c: Vec<u64> = cs.iter().flat_map(|c| c.data.iter().map(|x| x.as_canonical_u64())).collect();
        let mut out = vec![0u64; kappa * 54];
        let rc = unsafe {
            sys::neo_gpu_mix_rhos_commits(self.raw, r.as_ptr(), c.as_ptr(), cs.len() as u32, kappa as u32,
                                          out.as_mut_ptr())
        };
        self.check(rc).unwrap_or_else(|e| panic!("{e}"));
        Commitment { d: 54, kappa, data: out.into_iter().map(F::from_u64).collect() }
    }

    /// CommitMixers::combine_b_pows: sum_i b^(i-1) c_i (c_1 weight 1).
    pub fn combine_b_pows(&self, cs: &[Commitment], b: u32) -> Commitment {
        assert!(!cs.is_empty(), "combine_b_pows: no commitments");
        let kappa = cs[0].kappa;
        let c: Vec<u64> = cs.iter().flat_map(|c| c.data.iter().map(|x| x.as_canonical_u64())).collect();
        let mut out = vec![0u64; kappa * 54];
        let rc = unsafe {
            sys::neo_gpu_combine_b_pows(self.raw, c.as_ptr(), cs.len() as u32, kappa as u32, b, out.as_mut_ptr())
        };
        self.check(rc).unwrap_or_else(|e| panic!("{e}"));
        Commitment { d: 54, kappa, data: out.into_iter().map(F::from_u64).collect() }
    }
}

impl Drop for Context {
    fn drop(&mut self) {
        unsafe { sys::neo_gpu_ctx_destroy(self.raw) };
    }
}

/// A CCS structure in the library's layout (neo_ccs_desc): identity
/// sentinels, CSC matrices concatenated, f as (coeff, exponents) terms.
pub struct CcsDesc {
    n: u32,
    m: u32,
    t: u32,
    is_identity: Vec<u8>,
    col_ptr: Vec<u64>,
    nnz_off: Vec<u64>,
    row_idx: Vec<u32>,
    vals: Vec<u64>,
    f_coeff: Vec<u64>,
    f_exps: Vec<u32>,
}

impl CcsDesc {
    pub fn from_ccs(s: &CcsStructure<F>) -> Self {
        let t = s.matrices.len();
        let (mut is_identity, mut col_ptr, mut nnz_off) = (Vec::new(), Vec::new(), vec![0u64]);
        let (mut row_idx, mut vals) = (Vec::new(), Vec::new());
        for mat in &s.matrices {
            match mat {
                CcsMatrix::Identity { .. } => {
                    is_identity.push(1);
                    col_ptr.extend(core::iter::repeat(0u64).take(s.m + 1));
                }
                CcsMatrix::Csc(c) => {
                    is_identity.push(0);
                    col_ptr.extend(c.col_ptr.iter().map(|&p| p as u64));
                    row_idx.extend(c.row_idx.iter().map(|&r| r as u32));
                    vals.extend(c.vals.iter().map(|v| v.as_canonical_u64()));
                }
            }
            nnz_off.push(row_idx.len() as u64);
        }
        let mut f_coeff = Vec::new();
        let mut f_exps = Vec::new();
        for term in s.f.terms() {
            f_coeff.push(term.coeff.as_canonical_u64());
            f_exps.extend(term.exps.iter().copied());
        }
        Self { n: s.n as u32, m: s.m as u32, t: t as u32, is_identity, col_ptr, nnz_off, row_idx, vals, f_coeff, f_exps }
    }

    pub fn raw(&self) -> sys::neo_ccs_desc {
        sys::neo_ccs_desc {
            n: self.n,
            m: self.m,
            t: self.t,
            is_identity: self.is_identity.as_ptr(),
            col_ptr: self.col_ptr.as_ptr(),
            nnz_off: self.nnz_off.as_ptr(),
            row_idx: self.row_idx.as_ptr(),
            vals: self.vals.as_ptr(),
            n_terms: self.f_coeff.len() as u32,
            f_coeff: self.f_coeff.as_ptr(),
            f_exps: self.f_exps.as_ptr(),
        }
    }
}

/// Evaluations at `points` through `evals` (at most 16 points per call).
fn evals_chunked(points: &[K], mut evals: impl FnMut(&[u64], u32, &mut [u64]) -> i32, what: &str) -> Vec<K> {
    let mut out = Vec::with_capacity(points.len());
    for chunk in points.chunks(16) {
        let xs = flat_k(chunk);
        let mut ys = vec![0u64; 2 * chunk.len()];
        let rc = evals(&xs, chunk.len() as u32, &mut ys);
        if rc != 0 {
            panic!("neo-gpu {what}: evals failed with status {rc}");
        }
        out.extend(ys.chunks(2).map(k_from));
    }
    out
}

/// Pi_CCS RoundOracle on the GPU (OptimizedOracle, crates/neo-reductions/src/
/// engines/optimized_engine/oracle.rs): ell_n row rounds then ell_d Ajtai rounds.
pub struct GpuCcsOracle<'c> {
    ctx: &'c Context,
    raw: *mut sys::neo_gpu_ccs_oracle,
}

impl<'c> GpuCcsOracle<'c> {
    /// zs: the k digit matrices (54 x m) of the MCS witness and the carried
    /// ME witnesses; challenges as in oracle.rs:82-135.
    #[allow(clippy::too_many_arguments)]
    pub fn new(ctx: &'c Context, ccs: &CcsDesc, zs: &[Mat<F>], b: u32, alpha: &[K], beta_a: &[K], beta_r: &[K],
               gamma: K, r_inputs: Option<&[K]>, ell_d: u32, ell_n: u32, d_sc: u32) -> Result<Self> {
        let digits: Vec<i8> = zs.iter().flat_map(digits_i8).collect();
        let desc = ccs.raw();
        let (al, ba, br, g) = (flat_k(alpha), flat_k(beta_a), flat_k(beta_r), k_words(&gamma));
        let ri = r_inputs.map(flat_k);
        let mut raw = core::ptr::null_mut();
        let rc = unsafe {
            sys::neo_gpu_ccs_oracle_create(ctx.raw, &desc, digits.as_ptr(), zs.len() as u32, b, al.as_ptr(),
                                           ba.as_ptr(), br.as_ptr(), g.as_ptr(),
                                           ri.as_ref().map_or(core::ptr::null(), |v| v.as_ptr()), ell_d, ell_n,
                                           d_sc, &mut raw)
        };
        ctx.check(rc)?;
        Ok(Self { ctx, raw })
    }

    /// y (k x t x 54 K) and y_scalars (k x t K) of the ME outputs after all rounds.
    pub fn me_outputs(&mut self, k: usize, t: usize) -> Result<(Vec<K>, Vec<K>)> {
        let mut y = vec![0u64; k * t * 54 * 2];
        let mut ys = vec![0u64; k * t * 2];
        self.ctx.check(unsafe { sys::neo_gpu_ccs_oracle_me_outputs(self.raw, y.as_mut_ptr(), ys.as_mut_ptr()) })?;
        Ok((y.chunks(2).map(k_from).collect(), ys.chunks(2).map(k_from).collect()))
    }
}

impl RoundOracle for GpuCcsOracle<'_> {
    fn evals_at(&mut self, points: &[K]) -> Vec<K> {
        let raw = self.raw;
        evals_chunked(points, |xs, n, ys| unsafe { sys::neo_gpu_ccs_oracle_evals(raw, xs.as_ptr(), n, ys.as_mut_ptr()) },
                      "ccs oracle")
    }
    fn num_rounds(&self) -> usize {
        unsafe { sys::neo_gpu_ccs_oracle_num_rounds(self.raw) as usize }
    }
    fn degree_bound(&self) -> usize {
        unsafe { sys::neo_gpu_ccs_oracle_degree_bound(self.raw) as usize }
    }
    fn fold(&mut self, r: K) {
        let w = k_words(&r);
        let rc = unsafe { sys::neo_gpu_ccs_oracle_fold(self.raw, w.as_ptr()) };
        self.ctx.check(rc).unwrap_or_else(|e| panic!("{e}"));
    }
}

impl Drop for GpuCcsOracle<'_> {
    fn drop(&mut self) {
        unsafe { sys::neo_gpu_ccs_oracle_destroy(self.raw) };
    }
}

/// A Twist / Shout time-lane oracle (kind = sys::NEO_MEM_*) over dense
/// columns (2^ell K rows each, in the order include/neo_gpu.h lists per kind).
pub struct GpuMemOracle<'c> {
    ctx: &'c Context,
    raw: *mut sys::neo_gpu_mem_oracle,
    claim: K,
}

impl<'c> GpuMemOracle<'c> {
    #[allow(clippy::too_many_arguments)]
    pub fn new(ctx: &'c Context, kind: i32, ell: u32, r_point: Option<&[K]>, ell_addr: u32, r_addr: Option<&[K]>,
               init_at_r_addr: Option<K>, cols: &[Vec<K>], weights: Option<&[K]>) -> Result<Self> {
        let rp = r_point.map(flat_k);
        let ra = r_addr.map(flat_k);
        let ini = init_at_r_addr.map(|k| k_words(&k));
        let c: Vec<u64> = cols.iter().flat_map(|col| flat_k(col)).collect();
        let w = weights.map(flat_k);
        let mut claim = [0u64; 2];
        let mut raw = core::ptr::null_mut();
        let rc = unsafe {
            sys::neo_gpu_mem_oracle_create(ctx.raw, kind, ell, rp.as_ref().map_or(core::ptr::null(), |v| v.as_ptr()),
                                           ell_addr, ra.as_ref().map_or(core::ptr::null(), |v| v.as_ptr()),
                                           ini.as_ref().map_or(core::ptr::null(), |v| v.as_ptr()), cols.len() as u32,
                                           c.as_ptr(), w.as_ref().map_or(core::ptr::null(), |v| v.as_ptr()),
                                           claim.as_mut_ptr(), &mut raw)
        };
        ctx.check(rc)?;
        Ok(Self { ctx, raw, claim: k_from(&claim) })
    }

    /// The oracle's claimed sum over the hypercube (its round-0 p(0) + p(1)).
    pub fn claim(&self) -> K {
        self.claim
    }
}

impl RoundOracle for GpuMemOracle<'_> {
    fn evals_at(&mut self, points: &[K]) -> Vec<K> {
        let raw = self.raw;
        evals_chunked(points, |xs, n, ys| unsafe { sys::neo_gpu_mem_oracle_evals(raw, xs.as_ptr(), n, ys.as_mut_ptr()) },
                      "memory oracle")
    }
    fn num_rounds(&self) -> usize {
        unsafe { sys::neo_gpu_mem_oracle_num_rounds(self.raw) as usize }
    }
    fn degree_bound(&self) -> usize {
        unsafe { sys::neo_gpu_mem_oracle_degree_bound(self.raw) as usize }
    }
    fn fold(&mut self, r: K) {
        let w = k_words(&r);
        let rc = unsafe { sys::neo_gpu_mem_oracle_fold(self.raw, w.as_ptr()) };
        self.ctx.check(rc).unwrap_or_else(|e| panic!("{e}"));
    }
}

impl Drop for GpuMemOracle<'_> {
    fn drop(&mut self) {
        unsafe { sys::neo_gpu_mem_oracle_destroy(self.raw) };
    }
}

/// The Twist address-lane oracle (Read/WriteCheckAddrOracleSparseTime,
/// crates/neo-memory/src/twist_oracle.rs:1259-1642) from the instance's
/// columns and MemInit.
pub struct GpuTwistAddr<'c> {
    ctx: &'c Context,
    raw: *mut sys::neo_gpu_twist_addr,
}

impl<'c> GpuTwistAddr<'c> {
    #[allow(clippy::too_many_arguments)]
    pub fn new(ctx: &'c Context, kind: i32, ell: u32, r_cycle: &[K], ell_addr: u32, init: &[(u64, F)],
               cols: &[Vec<K>]) -> Result<Self> {
        let rc_ = flat_k(r_cycle);
        let ia: Vec<u64> = init.iter().map(|p| p.0).collect();
        let iv: Vec<u64> = init.iter().map(|p| p.1.as_canonical_u64()).collect();
        let c: Vec<u64> = cols.iter().flat_map(|col| flat_k(col)).collect();
        let mut raw = core::ptr::null_mut();
        let rc = unsafe {
            sys::neo_gpu_twist_addr_create(ctx.raw, kind, ell, rc_.as_ptr(), ell_addr, init.len() as u64,
                                           if init.is_empty() { core::ptr::null() } else { ia.as_ptr() },
                                           if init.is_empty() { core::ptr::null() } else { iv.as_ptr() },
                                           c.as_ptr(), &mut raw)
        };
        ctx.check(rc)?;
        Ok(Self { ctx, raw })
    }
}

impl RoundOracle for GpuTwistAddr<'_> {
    fn evals_at(&mut self, points: &[K]) -> Vec<K> {
        let raw = self.raw;
        evals_chunked(points, |xs, n, ys| unsafe { sys::neo_gpu_twist_addr_evals(raw, xs.as_ptr(), n, ys.as_mut_ptr()) },
                      "twist address oracle")
    }
    fn num_rounds(&self) -> usize {
        unsafe { sys::neo_gpu_twist_addr_num_rounds(self.raw) as usize }
    }
    fn degree_bound(&self) -> usize {
        unsafe { sys::neo_gpu_twist_addr_degree_bound(self.raw) as usize }
    }
    fn fold(&mut self, r: K) {
        let w = k_words(&r);
        let rc = unsafe { sys::neo_gpu_twist_addr_fold(self.raw, w.as_ptr()) };
        self.ctx.check(rc).unwrap_or_else(|e| panic!("{e}"));
    }
}

impl Drop for GpuTwistAddr<'_> {
    fn drop(&mut self) {
        unsafe { sys::neo_gpu_twist_addr_destroy(self.raw) };
    }
}

/// The Ajtai S-module homomorphism on the GPU for one registered PP (kappa, m):
/// `commit` runs the tensor-core commitment of a 54 x m digit matrix
/// (AjtaiSModule::commit, crates/neo-ajtai/src/s_module.rs:336-364).
pub struct GpuAjtai<'c> {
    pub ctx: &'c Context,
    pub kappa: u32,
}

impl SModuleHomomorphism<F, Commitment> for GpuAjtai<'_> {
    fn commit(&self, z: &Mat<F>) -> Commitment {
        assert_eq!(z.rows(), 54, "commit: Z must have d = 54 rows");
        let m = z.cols() as u64;
        let out = self.ctx.commit_digits(&digits_i8(z), 1, m, self.kappa).unwrap_or_else(|e| panic!("{e}"));
        Commitment { d: 54, kappa: self.kappa as usize, data: out.into_iter().map(F::from_u64).collect() }
    }

    fn project_x(&self, z: &Mat<F>, min: usize) -> Mat<F> {
        let mut data = Vec::with_capacity(z.rows() * min);
        for r in 0..z.rows() {
            data.extend_from_slice(&z.row(r)[..min]);
        }
        Mat::from_row_major(z.rows(), min, data)
    }
}
