// core.cu -- context, CCS upload, decomposition, Pi_RLC mix, Pi_DEC split and
// ME evaluations y = Z (M^T chi_r).
#include "internal.cuh"
#include <algorithm>

using gl::K;

static int neo_gpu_ctx_create_impl_abi(int device, neo_gpu_ctx** out) {
    if (!out) return NEO_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NEO_ERR_CUDA;
    if (device < 0 || device >= ndev) return NEO_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return NEO_ERR_CUDA;
    neo_gpu_ctx* c = new neo_gpu_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return NEO_ERR_CUDA;
    }
    if (cudaMalloc(&c->d_err, sizeof(uint32_t)) != cudaSuccess || cudaMemset(c->d_err, 0, sizeof(uint32_t)) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return NEO_ERR_CUDA;
    }
    *out = c;
    return NEO_OK;
}
extern "C" int neo_gpu_ctx_create(int device, neo_gpu_ctx** out) { NEO_ABI_GUARD(neo_gpu_ctx_create_impl_abi(device, out)) }

// Stream on which DevBuf allocations of this thread are made (stream-ordered,
// from the device's memory pool) and later freed; null: cudaMalloc / cudaFree.
thread_local cudaStream_t g_alloc_stream = nullptr;

static int neo_gpu_ctx_destroy_impl_abi(neo_gpu_ctx* ctx) {
    if (!ctx) return NEO_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->chi_cache) cudaFree(ctx->chi_cache);
    if (ctx->d_err) cudaFree(ctx->d_err);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return NEO_OK;
}
extern "C" int neo_gpu_ctx_destroy(neo_gpu_ctx* ctx) { NEO_ABI_GUARD(neo_gpu_ctx_destroy_impl_abi(ctx)) }

extern "C" const char* neo_gpu_last_error(const neo_gpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
extern "C" uint64_t neo_gpu_kernel_launches(const neo_gpu_ctx* ctx) { return ctx ? ctx->launches : 0; }
int check_device_error(neo_gpu_ctx* ctx) {
    uint32_t e = 0;
    NEO_CK(ctx, ctx_d2h(ctx, &e, ctx->d_err, 4));
    NEO_CK(ctx, ctx_sync(ctx));
    if (e) {
        NEO_CK(ctx, cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream));
        char buf[128];
        if (e == (1u << 16)) {  // set by the small-digit commitment form only
            snprintf(buf, sizeof buf, "commitment digits outside [-63, 63] on the small-digit path");
            return ctx->fail(NEO_ERR_INVARIANT, buf);
        }
        snprintf(buf, sizeof buf, "device wait timed out (error bits 0x%x)", e);
        return ctx->fail(NEO_ERR_CUDA, buf);
    }
    return NEO_OK;
}

// Bounded device wait: one thread polls *flag up to `limit` times (about
// 1 us apart); a wait that runs out sets bit 0x10 of the context's error word
// and returns, like the commitment kernel's bounded mbarrier waits.
__global__ void wait_flag_kernel(const volatile uint32_t* flag, uint32_t limit, uint32_t* err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (uint32_t it = 0; it < limit; it++) {
        if (*flag) return;
        __nanosleep(1000);
    }
    atomicOr(err, 0x10u);
}

static int neo_gpu_wait_probe_impl_abi(neo_gpu_ctx* ctx, uint32_t set_flag, uint32_t spin_limit) {
    if (!ctx) return NEO_ERR_ARG;
    if (spin_limit == 0 || spin_limit > (1u << 20)) return ctx->fail(NEO_ERR_ARG, "wait_probe: spin_limit in [1, 2^20]");
    cudaSetDevice(ctx->device);
    DevBuf<uint32_t> flag;
    NEO_CK(ctx, flag.alloc(1));
    NEO_CK(ctx, cudaMemsetAsync(flag.p, 0, 4, ctx->stream));
    if (set_flag) NEO_CK(ctx, cudaMemsetAsync(flag.p, 0xFF, 4, ctx->stream));
    wait_flag_kernel<<<1, 32, 0, ctx->stream>>>(flag.p, spin_limit, ctx->d_err);
    NEO_LAUNCHED(ctx);
    return check_device_error(ctx);  // synchronizes; a timeout is reported and cleared
}
extern "C" int neo_gpu_wait_probe(neo_gpu_ctx* ctx, uint32_t set_flag, uint32_t spin_limit) { NEO_ABI_GUARD(neo_gpu_wait_probe_impl_abi(ctx, set_flag, spin_limit)) }

static int neo_gpu_ctx_stream_impl_abi(const neo_gpu_ctx* ctx, void** stream) {
    if (!ctx || !stream) return NEO_ERR_ARG;
    *stream = (void*)ctx->stream;
    return NEO_OK;
}
extern "C" int neo_gpu_ctx_stream(const neo_gpu_ctx* ctx, void** stream) { NEO_ABI_GUARD(neo_gpu_ctx_stream_impl_abi(ctx, stream)) }
static int neo_gpu_synchronize_impl_abi(neo_gpu_ctx* ctx) {
    if (!ctx) return NEO_ERR_ARG;
    cudaSetDevice(ctx->device);
    return check_device_error(ctx);  // waits for the stream, then reports (and clears) device-side errors
}
extern "C" int neo_gpu_synchronize(neo_gpu_ctx* ctx) { NEO_ABI_GUARD(neo_gpu_synchronize_impl_abi(ctx)) }

// ---------------------------------------------------------------------------
// CCS upload: CSC as given, plus a CSR copy built on the host.
// ---------------------------------------------------------------------------
int dev_ccs_upload(neo_gpu_ctx* ctx, const neo_ccs_desc* d, DevCcs& o) {
    if (!d || d->t == 0 || d->m == 0 || d->n == 0 || d->t > 16 || d->n_terms == 0 || d->n_terms > 16)
        return ctx->fail(NEO_ERR_ARG, "ccs: bad dimensions");
    o.n = d->n; o.m = d->m; o.t = d->t; o.n_terms = d->n_terms;
    o.is_identity.assign(d->is_identity, d->is_identity + d->t);
    o.f_coeff.assign(d->f_coeff, d->f_coeff + d->n_terms);
    o.f_exps.assign(d->f_exps, d->f_exps + (size_t)d->n_terms * d->t);
    o.nnz_off.assign(d->nnz_off, d->nnz_off + d->t + 1);
    uint64_t nnz = o.nnz_off[d->t];
    std::vector<uint64_t> csr_ptr((size_t)d->t * (d->n + 1), 0);
    std::vector<uint32_t> csr_col(std::max<uint64_t>(nnz, 1));
    std::vector<uint64_t> csr_val(std::max<uint64_t>(nnz, 1));
    for (uint32_t j = 0; j < d->t; j++) {
        if (o.is_identity[j]) continue;
        const uint64_t* cp = d->col_ptr + (size_t)j * (d->m + 1);
        uint64_t base = o.nnz_off[j];
        uint64_t cnt = o.nnz_off[j + 1] - base;
        if (cp[d->m] != cnt) return ctx->fail(NEO_ERR_ARG, "ccs: col_ptr inconsistent with nnz_off");
        uint64_t* rp = csr_ptr.data() + (size_t)j * (d->n + 1);
        for (uint64_t k = 0; k < cnt; k++) {
            uint32_t r = d->row_idx[base + k];
            if (r >= d->n) return ctx->fail(NEO_ERR_ARG, "ccs: row index out of range");
            rp[r + 1]++;
        }
        for (uint32_t r = 0; r < d->n; r++) rp[r + 1] += rp[r];
        std::vector<uint64_t> fill(rp, rp + d->n);
        for (uint32_t c = 0; c < d->m; c++)
            for (uint64_t k = cp[c]; k < cp[c + 1]; k++) {
                uint32_t r = d->row_idx[base + k];
                uint64_t pos = base + fill[r]++;
                csr_col[pos] = c;
                csr_val[pos] = gl::canon(d->vals[base + k]);
            }
    }
    size_t nn = std::max<uint64_t>(nnz, 1);
    NEO_CK(ctx, o.csr_ptr.alloc(csr_ptr.size()));
    NEO_CK(ctx, o.csr_col.alloc(nn));
    NEO_CK(ctx, o.csr_val.alloc(nn));
    NEO_CK(ctx, o.csc_ptr.alloc((size_t)d->t * (d->m + 1)));
    NEO_CK(ctx, o.csc_row.alloc(nn));
    NEO_CK(ctx, o.csc_val.alloc(nn));
    NEO_CK(ctx, cudaMemcpyAsync(o.csr_ptr.p, csr_ptr.data(), csr_ptr.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(o.csr_col.p, csr_col.data(), nn * 4, cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(o.csr_val.p, csr_val.data(), nn * 8, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<uint64_t> csc_ptr((size_t)d->t * (d->m + 1), 0);
    for (uint32_t j = 0; j < d->t; j++)
        if (!o.is_identity[j]) memcpy(&csc_ptr[(size_t)j * (d->m + 1)], d->col_ptr + (size_t)j * (d->m + 1), (d->m + 1) * 8);
    std::vector<uint64_t> csc_val(nn, 0);
    if (nnz) for (uint64_t k = 0; k < nnz; k++) csc_val[k] = gl::canon(d->vals[k]);
    NEO_CK(ctx, cudaMemcpyAsync(o.csc_ptr.p, csc_ptr.data(), csc_ptr.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (nnz) {
        NEO_CK(ctx, cudaMemcpyAsync(o.csc_row.p, d->row_idx, nnz * 4, cudaMemcpyHostToDevice, ctx->stream));
        NEO_CK(ctx, cudaMemcpyAsync(o.csc_val.p, csc_val.data(), nnz * 8, cudaMemcpyHostToDevice, ctx->stream));
    }
    return NEO_OK;
}

// ---------------------------------------------------------------------------
// chi table: w[mask] = prod_i (bit_i(mask) ? b_i : 1 - b_i)
// (crates/neo-reductions/src/engines/optimized_engine/oracle.rs:1525-1540)
// ---------------------------------------------------------------------------
__global__ void chi_table_kernel(const K* __restrict__ bits, uint32_t nbits, K* __restrict__ out) {
    uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (idx >= (1ULL << nbits)) return;
    K w = gl::kone();
    for (uint32_t i = 0; i < nbits; i++) {
        K b = bits[i];
        w = gl::kmul(w, ((idx >> i) & 1) ? b : gl::ksub(gl::kone(), b));
    }
    out[idx] = w;
}

int launch_chi_table(neo_gpu_ctx* ctx, const K* d_bits, uint32_t nbits, K* d_out) {
    uint64_t len = 1ULL << nbits;
    chi_table_kernel<<<ceil_div(len, 256), 256, 0, ctx->stream>>>(d_bits, nbits, d_out);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}

// The tables chi(bits[j+1..nbits)) of every j < nbits in one launch: table j
// (2^(nbits-j-1) entries) sits at n - n/2^j, n = 2^nbits, so an index's
// leading one bits give its j.
__global__ void suffix_chi_kernel(const K* __restrict__ bits, uint32_t nbits, K* __restrict__ out) {
    const uint64_t n = 1ULL << nbits;
    const uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (idx + 1 >= n) return;
    const uint32_t j = __clzll(~(idx << (64 - nbits)));  // leading ones of the nbits-bit index
    const uint64_t local = idx - (n - (n >> j));
    K w = gl::kone();
    for (uint32_t i = 0; i + j + 1 < nbits; i++) {
        const K b = bits[j + 1 + i];
        w = gl::kmul(w, ((local >> i) & 1) ? b : gl::ksub(gl::kone(), b));
    }
    out[idx] = w;
}

int launch_suffix_chi_tables(neo_gpu_ctx* ctx, const K* d_bits, uint32_t nbits, K* d_out) {
    if (nbits == 0) return NEO_OK;
    const uint64_t n = 1ULL << nbits;
    suffix_chi_kernel<<<ceil_div(n - 1, 256), 256, 0, ctx->stream>>>(d_bits, nbits, d_out);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}

// ---------------------------------------------------------------------------
// decomp_b (b = 2, balanced) (crates/neo-ajtai/src/decomp.rs:118-158)
// ---------------------------------------------------------------------------
__global__ void decomp_b2_kernel(const uint64_t* __restrict__ z, uint64_t m, int8_t* __restrict__ Z) {
    uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c >= m) return;
    uint64_t u = gl::canon(z[c]);
    const uint64_t half = (GL_Q - 1) / 2;
    int64_t a = u <= half ? (int64_t)u : -(int64_t)(GL_Q - u);
#pragma unroll
    for (int row = 0; row < NEO_D; row++) {
        int64_t digit = (a & 1) == 0 ? 0 : (a >= 0 ? 1 : -1);
        Z[(uint64_t)row * m + c] = (int8_t)digit;
        a = (a - digit) >> 1;
    }
}

static int neo_gpu_decomp_b2_impl_abi(neo_gpu_ctx* ctx, const uint64_t* z, uint64_t m, int8_t* Z) {
    if (!ctx || !z || !Z || m == 0) return ctx ? ctx->fail(NEO_ERR_ARG, "decomp: bad args") : NEO_ERR_ARG;
    cudaSetDevice(ctx->device);
    DevBuf<uint64_t> dz;
    DevBuf<int8_t> dZ;
    NEO_CK(ctx, dz.alloc(m));
    NEO_CK(ctx, dZ.alloc((size_t)NEO_D * m));
    NEO_CK(ctx, cudaMemcpyAsync(dz.p, z, m * 8, cudaMemcpyHostToDevice, ctx->stream));
    decomp_b2_kernel<<<ceil_div(m, 256), 256, 0, ctx->stream>>>(dz.p, m, dZ.p);
    NEO_LAUNCHED(ctx);
    NEO_CK(ctx, ctx_d2h(ctx, Z, dZ.p, (size_t)NEO_D * m));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_decomp_b2(neo_gpu_ctx* ctx, const uint64_t* z, uint64_t m, int8_t* Z) { NEO_ABI_GUARD(neo_gpu_decomp_b2_impl_abi(ctx, z, m, Z)) }

// ---------------------------------------------------------------------------
// Pi_RLC mix: Z_mix[:, c] = sum_i a_i(X) z_{i,c}(X) mod Phi_81 over the
// integers (all entries are small, so this equals the F_q computation of
// optimized_engine/common.rs:1221-1379 with rot_from_coeffs common.rs:398-430).
// Zmix = [rot_1 .. rot_k] (54 x 54k) times the stacked digit planes
// (54k x m), exact in int32.  Each thread owns one column and RPT of the 54
// output rows (small m uses fewer rows per thread so the grid still covers
// the SMs).  Per input it issues the column's 54 digit loads together (one
// memory latency per input instead of one per digit), packs them four to a
// word and multiplies with dp4a against the rot rows, which sit in shared
// memory as int8 rows padded to RLC_ROT_ROW = 64 bytes (zeros past k = 54)
// and are read 16 bytes at a time.  Any split gives the same Zmix.
// ---------------------------------------------------------------------------
template <int RPT>
__global__ void __launch_bounds__(128) rlc_mix_kernel(const int8_t* __restrict__ rot, const int8_t* __restrict__ Zs,
                                                      uint32_t count, uint64_t m, int32_t* __restrict__ Zmix) {
    extern __shared__ int4 s_rot[];  // [count][54][64 B]
    const uint32_t n16 = count * NEO_D * (RLC_ROT_ROW / 16);
    const int4* g = reinterpret_cast<const int4*>(rot);
    for (uint32_t x = threadIdx.x; x < n16; x += blockDim.x) s_rot[x] = g[x];
    __syncthreads();
    const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const int r0 = blockIdx.y * RPT;
    if (c >= m) return;
    int32_t acc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) acc[r] = 0;
    for (uint32_t i = 0; i < count; i++) {
        const int8_t* Zi = Zs + (uint64_t)i * NEO_D * m + c;
        uint32_t zb[NEO_D];
#pragma unroll
        for (int k = 0; k < NEO_D; k++) zb[k] = (uint8_t)Zi[(uint64_t)k * m];
        int w[14];  // bytes 4j..4j+3 of the column (k = 54, 55 are zero)
#pragma unroll
        for (int j = 0; j < 13; j++) w[j] = (int)(zb[4 * j] | (zb[4 * j + 1] << 8) | (zb[4 * j + 2] << 16) | (zb[4 * j + 3] << 24));
        w[13] = (int)(zb[52] | (zb[53] << 8));
        const int4* R = s_rot + ((uint64_t)i * NEO_D + r0) * (RLC_ROT_ROW / 16);
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            const int4 q0 = R[4 * r], q1 = R[4 * r + 1], q2 = R[4 * r + 2], q3 = R[4 * r + 3];
            int a = acc[r];
            a = __dp4a(w[0], q0.x, a); a = __dp4a(w[1], q0.y, a); a = __dp4a(w[2], q0.z, a); a = __dp4a(w[3], q0.w, a);
            a = __dp4a(w[4], q1.x, a); a = __dp4a(w[5], q1.y, a); a = __dp4a(w[6], q1.z, a); a = __dp4a(w[7], q1.w, a);
            a = __dp4a(w[8], q2.x, a); a = __dp4a(w[9], q2.y, a); a = __dp4a(w[10], q2.z, a); a = __dp4a(w[11], q2.w, a);
            a = __dp4a(w[12], q3.x, a); a = __dp4a(w[13], q3.y, a);  // q3.z, q3.w: the row's zero padding
            acc[r] = a;
        }
    }
#pragma unroll
    for (int r = 0; r < RPT; r++) Zmix[(uint64_t)(r0 + r) * m + c] = acc[r];
}

// integer rot(a): column t = a X^t mod Phi_81 (commit.rs:46-54 recurrence)
static void rot_int8(const int8_t* a, int8_t* out) {
    int32_t col[NEO_D], nxt[NEO_D];
    for (int r = 0; r < NEO_D; r++) col[r] = a[r];
    for (int t = 0; t < NEO_D; t++) {
        for (int r = 0; r < NEO_D; r++) out[r * NEO_D + t] = (int8_t)col[r];
        int32_t last = col[NEO_D - 1];
        nxt[0] = -last;
        for (int q = 1; q < NEO_D; q++) nxt[q] = col[q - 1];
        nxt[27] -= last;
        memcpy(col, nxt, sizeof col);
    }
}

int rlc_mix_device(neo_gpu_ctx* ctx, const int8_t* rho_coeffs_host, const int8_t* d_Zs, uint32_t count, uint64_t m,
                   int32_t* d_Zmix, int8_t* d_rot_scratch) {
    std::vector<int8_t> rot((size_t)count * NEO_D * NEO_D);
    for (uint32_t i = 0; i < count; i++) {
        for (int r = 0; r < NEO_D; r++)
            if (rho_coeffs_host[i * NEO_D + r] < -2 || rho_coeffs_host[i * NEO_D + r] > 2)
                return ctx->fail(NEO_ERR_ARG, "rlc: rho coefficient outside {-2..2}");
        if (count == 1) {
            memset(rot.data(), 0, NEO_D * NEO_D);
            for (int r = 0; r < NEO_D; r++) rot[r * NEO_D + r] = 1;  // identity (common.rs:560-564)
        } else {
            rot_int8(rho_coeffs_host + i * NEO_D, rot.data() + (size_t)i * NEO_D * NEO_D);
        }
    }
    // rows padded to RLC_ROT_ROW bytes for the kernel's 16-byte shared loads
    std::vector<int8_t> rot_pad((size_t)count * NEO_D * RLC_ROT_ROW, 0);
    for (size_t row = 0; row < (size_t)count * NEO_D; row++)
        memcpy(&rot_pad[row * RLC_ROT_ROW], &rot[row * NEO_D], NEO_D);
    NEO_CK(ctx, cudaMemcpyAsync(d_rot_scratch, rot_pad.data(), rot_pad.size(), cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, ctx_sync(ctx));  // rot_pad is pageable host memory that goes away on return
    size_t smem = rot_pad.size();
    // rows per thread: the most that still gives two waves of blocks over the SMs
    const unsigned col_blocks = ceil_div(m, 128);
    auto launch = [&](auto kernel, int rpt) -> int {
        static SmemLimit limit[4];
        SmemLimit& l = limit[rpt == 54 ? 0 : rpt == 18 ? 1 : rpt == 6 ? 2 : 3];
        if (smem > 48 * 1024) NEO_CK(ctx, l.at_least(kernel, smem));
        kernel<<<dim3(col_blocks, NEO_D / rpt), 128, smem, ctx->stream>>>(d_rot_scratch, d_Zs, count, m, d_Zmix);
        NEO_LAUNCHED(ctx);
        return NEO_OK;
    };
    const unsigned want = 2 * 148;
    if (col_blocks >= want) return launch(rlc_mix_kernel<54>, 54);
    if (col_blocks * 3 >= want) return launch(rlc_mix_kernel<18>, 18);
    if (col_blocks * 9 >= want) return launch(rlc_mix_kernel<6>, 6);
    return launch(rlc_mix_kernel<1>, 1);
}

static int neo_gpu_rlc_mix_impl_abi(neo_gpu_ctx* ctx, const int8_t* rho_coeffs, const int8_t* Zs, uint32_t count,
                               uint64_t m, int32_t* Zmix) {
    if (!ctx) return NEO_ERR_ARG;
    if (!rho_coeffs || !Zs || !Zmix || count == 0 || count > 64 || m == 0) return ctx->fail(NEO_ERR_ARG, "rlc: bad args");
    cudaSetDevice(ctx->device);
    DevBuf<int8_t> dZs, drot;
    DevBuf<int32_t> dmix;
    NEO_CK(ctx, dZs.alloc((size_t)count * NEO_D * m));
    NEO_CK(ctx, drot.alloc((size_t)count * NEO_D * RLC_ROT_ROW));
    NEO_CK(ctx, dmix.alloc((size_t)NEO_D * m));
    NEO_CK(ctx, cudaMemcpyAsync(dZs.p, Zs, dZs.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    int rc = rlc_mix_device(ctx, rho_coeffs, dZs.p, count, m, dmix.p, drot.p);
    if (rc) return rc;
    NEO_CK(ctx, ctx_d2h(ctx, Zmix, dmix.p, dmix.bytes()));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_rlc_mix(neo_gpu_ctx* ctx, const int8_t* rho_coeffs, const int8_t* Zs, uint32_t count,
                               uint64_t m, int32_t* Zmix) { NEO_ABI_GUARD(neo_gpu_rlc_mix_impl_abi(ctx, rho_coeffs, Zs, count, m, Zmix)) }

// ---------------------------------------------------------------------------
// Pi_DEC split (common.rs:75-268; balanced_divrem common.rs:44-58)
// flags[0] = out-of-range error, flags[1 + i] = plane i nonzero
// ---------------------------------------------------------------------------
// Z_mix entries are int32, so the digits come from 32-bit arithmetic; b = 2
// (the fold step's base) takes the balanced remainder and an exact shift
// instead of a division.
template <bool B2>
__global__ void split_b_kernel(const int32_t* __restrict__ Zmix, uint64_t len, uint32_t k, int32_t b,
                               int8_t* __restrict__ planes, uint32_t* __restrict__ flags) {
    uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint32_t nz_mask = 0;
    if (idx < len) {
        int32_t v = Zmix[idx];
        // b^k, saturated once it exceeds every int32 (the check is then moot)
        int64_t B = 1;
        for (uint32_t i = 0; i < k && B <= INT32_MAX; i++) B *= b;
        if ((int64_t)v >= B || (int64_t)v <= -B) atomicOr(&flags[0], 1u);
        const int32_t half = b / 2;
        for (uint32_t i = 0; i < k; i++) {
            int32_t r, q;
            if (B2) {  // v % 2 in {-1, 0, 1} (sign of v), v - r even
                r = (v & 1) ? (v < 0 ? -1 : 1) : 0;
                q = (v - r) >> 1;
            } else {
                r = v % b;
                q = (v - r) / b;
                if (r > half) { r -= b; q += 1; }
                else if (r < -half) { r += b; q -= 1; }
            }
            planes[(uint64_t)i * len + idx] = (int8_t)r;
            if (r) nz_mask |= 1u << i;
            v = q;
        }
        if (v != 0) atomicOr(&flags[0], 1u);
    }
    // block-aggregate the nonzero plane mask; one atomic per block, and none
    // once every plane it saw is already flagged (a single address that every
    // warp hit serialised the kernel)
    for (int o = 16; o > 0; o >>= 1) nz_mask |= __shfl_xor_sync(0xffffffffu, nz_mask, o);
    __shared__ uint32_t s_mask;
    if (threadIdx.x == 0) s_mask = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && nz_mask) atomicOr(&s_mask, nz_mask);
    __syncthreads();
    if (threadIdx.x == 0 && s_mask && (s_mask & ~__ldcg(flags + 1))) atomicOr(&flags[1], s_mask);
}

int split_b_device(neo_gpu_ctx* ctx, const int32_t* d_Zmix, uint64_t len, uint32_t k, uint32_t b, int8_t* d_planes,
                   uint32_t* d_flags) {
    if (k == 0 || k > 31 || b < 2 || b > 64) return ctx->fail(NEO_ERR_UNSUPPORTED, "split_b: k/b out of range");
    NEO_CK(ctx, cudaMemsetAsync(d_flags, 0, 2 * sizeof(uint32_t), ctx->stream));
    if (b == 2)
        split_b_kernel<true><<<ceil_div(len, 256), 256, 0, ctx->stream>>>(d_Zmix, len, k, 2, d_planes, d_flags);
    else
        split_b_kernel<false><<<ceil_div(len, 256), 256, 0, ctx->stream>>>(d_Zmix, len, k, (int32_t)b, d_planes, d_flags);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}

static int neo_gpu_split_b_impl_abi(neo_gpu_ctx* ctx, const int32_t* Zmix, uint64_t len, uint32_t k, uint32_t b,
                               int8_t* planes, uint8_t* nonzero) {
    if (!ctx) return NEO_ERR_ARG;
    if (!Zmix || !planes || !nonzero || len == 0) return ctx->fail(NEO_ERR_ARG, "split_b: bad args");
    cudaSetDevice(ctx->device);
    DevBuf<int32_t> dmix;
    DevBuf<int8_t> dpl;
    DevBuf<uint32_t> dfl;
    NEO_CK(ctx, dmix.alloc(len));
    NEO_CK(ctx, dpl.alloc((size_t)k * len));
    NEO_CK(ctx, dfl.alloc(2));
    NEO_CK(ctx, cudaMemcpyAsync(dmix.p, Zmix, len * 4, cudaMemcpyHostToDevice, ctx->stream));
    int rc = split_b_device(ctx, dmix.p, len, k, b, dpl.p, dfl.p);
    if (rc) return rc;
    uint32_t flags[2];
    NEO_CK(ctx, ctx_d2h(ctx, flags, dfl.p, 8));
    NEO_CK(ctx, ctx_d2h(ctx, planes, dpl.p, (size_t)k * len));
    NEO_CK(ctx, ctx_sync(ctx));
    if (flags[0]) return ctx->fail(NEO_ERR_INVARIANT, "DEC split: entry out of range for k_rho digits");
    for (uint32_t i = 0; i < k; i++) nonzero[i] = (flags[1] >> i) & 1;
    return NEO_OK;
}
extern "C" int neo_gpu_split_b(neo_gpu_ctx* ctx, const int32_t* Zmix, uint64_t len, uint32_t k, uint32_t b,
                               int8_t* planes, uint8_t* nonzero) { NEO_ABI_GUARD(neo_gpu_split_b_impl_abi(ctx, Zmix, len, k, b, planes, nonzero)) }

// ---------------------------------------------------------------------------
// ME evaluations: v_j = M_j^T chi_r (CSC), y[w][j][rho] = sum_c Z_w[rho][c] v_j[c]
// (crates/neo-reductions/src/common.rs:582-650; oracle.rs:1694-1768)
// ---------------------------------------------------------------------------
__global__ void matT_chi_kernel(const uint64_t* __restrict__ csc_ptr, const uint32_t* __restrict__ csc_row,
                                const uint64_t* __restrict__ csc_val, int is_identity, uint32_t n, uint32_t m,
                                uint64_t n_sz, const K* __restrict__ chi, K* __restrict__ v) {
    uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c >= m) return;
    uint64_t n_eff = n < n_sz ? n : n_sz;
    if (is_identity) {
        v[c] = c < n_eff ? chi[c] : gl::kzero();
        return;
    }
    K acc = gl::kzero();
    for (uint64_t k = csc_ptr[c]; k < csc_ptr[c + 1]; k++) {
        uint32_t r = csc_row[k];
        if (r < n_eff) acc = gl::kadd(acc, gl::kscale(chi[r], csc_val[k]));
    }
    v[c] = acc;
}

// one block per (w, rho); threads stride over columns; t accumulators.
template <int TMAX>
__global__ void __launch_bounds__(256) zv_dot_kernel(const int8_t* __restrict__ Z, uint64_t m, uint32_t t,
                                                     const K* __restrict__ v, K* __restrict__ y) {
    const uint32_t row = blockIdx.x;  // w*54 + rho
    const int8_t* zr = Z + (uint64_t)row * m;
    K acc[TMAX];
#pragma unroll
    for (int j = 0; j < TMAX; j++) acc[j] = gl::kzero();
    for (uint64_t c = threadIdx.x; c < m; c += blockDim.x) {
        int z = zr[c];
        if (z == 0) continue;
#pragma unroll
        for (int j = 0; j < TMAX; j++) {
            if (j < (int)t) {
                K x = v[(uint64_t)j * m + c];
                acc[j] = z == 1 ? gl::kadd(acc[j], x) : (z == -1 ? gl::ksub(acc[j], x) : gl::kadd(acc[j], gl::kscale_small(x, z)));
            }
        }
    }
    __shared__ K red[TMAX][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < TMAX; j++) {
        K a = acc[j];
        for (int o = 16; o > 0; o >>= 1) {
            K b;
            b.re = __shfl_xor_sync(0xffffffffu, a.re, o);
            b.im = __shfl_xor_sync(0xffffffffu, a.im, o);
            a = gl::kadd(a, b);
        }
        if (lane == 0) red[j][warp] = a;
    }
    __syncthreads();
    if (threadIdx.x < t) {
        K a = gl::kzero();
        for (int wv = 0; wv < (int)(blockDim.x >> 5); wv++) a = gl::kadd(a, red[threadIdx.x][wv]);
        // y layout [w][t][54]
        uint32_t w = row / NEO_D, rho = row % NEO_D;
        y[((uint64_t)w * t + threadIdx.x) * NEO_D + rho] = a;
    }
}

// y[row][j] = sum_c Z[row][c] v[j][c] for ternary digit rows (the ME
// outputs y = Z M_j^T chi_r of compute_y_from_Z_and_r,
// crates/neo-reductions/src/common.rs:582-650, for many rows at once).  A
// block holds 128 rows (one per thread) and a range of columns; per chunk of
// 64 columns the 9 signed sums (d0 v[c] + d1 v[c+1], d in {-1,0,1}) of every
// column pair are tabulated in shared memory once for the block's rows, and a
// row adds one table entry per pair (index from its two digits), summed
// unreduced in 128 bits.  v is read once per 128 rows instead of once per row.
// Each block adds its column range's sums into per-(row, j) 64-bit
// accumulators with atomics (a wrap past 2^64 counted apart: exact and
// order-free), so the last block of a row group (ticket) only reduces them,
// instead of summing every column range's partial one after the other.
constexpr int ZR_ROWS = 128, ZR_CHUNK = 64, ZR_TMAX = 4;
constexpr int ZR_TPAD = 5;  // entry stride 80 B: the 9 entries of a pair fall on distinct bank groups
__global__ void __launch_bounds__(ZR_ROWS) zrows_kernel(const int8_t* __restrict__ Z, uint32_t R, uint64_t m,
                                                        uint32_t t, const K* __restrict__ v, uint64_t cols_per_split,
                                                        unsigned long long* __restrict__ acc_lo,
                                                        unsigned int* __restrict__ acc_wrap,
                                                        unsigned int* __restrict__ tickets, K* __restrict__ y) {
    __shared__ K tab[ZR_CHUNK / 2][9][ZR_TPAD];
    const uint32_t row = blockIdx.x * ZR_ROWS + threadIdx.x;
    const uint64_t c_lo = blockIdx.y * cols_per_split, c_hi = min(m, c_lo + cols_per_split);
    uint64_t lo[2 * ZR_TMAX], hi[2 * ZR_TMAX];
#pragma unroll
    for (int i = 0; i < 2 * ZR_TMAX; i++) lo[i] = hi[i] = 0;
    for (uint64_t c0 = c_lo; c0 < c_hi; c0 += ZR_CHUNK) {
        const uint32_t np = (uint32_t)(min((uint64_t)ZR_CHUNK, c_hi - c0) / 2);  // column pairs of this chunk
        __syncthreads();  // the previous chunk's table is no longer read
        for (uint32_t i = threadIdx.x; i < np * 9 * t; i += ZR_ROWS) {
            const uint32_t j = i % t, e = (i / t) % 9, g = i / (9 * t);
            const K a = v[(uint64_t)j * m + c0 + 2 * g], b = v[(uint64_t)j * m + c0 + 2 * g + 1];
            const uint32_t d0 = e % 3, d1 = e / 3;  // digit + 1
            K s = d0 == 0 ? gl::kneg(a) : (d0 == 2 ? a : gl::kzero());
            s = d1 == 0 ? gl::ksub(s, b) : (d1 == 2 ? gl::kadd(s, b) : s);
            tab[g][e][j] = s;
        }
        __syncthreads();
        if (row >= R) continue;
        const uint4* zr = reinterpret_cast<const uint4*>(Z + (uint64_t)row * m + c0);
        for (uint32_t g0 = 0; g0 < np; g0 += 8) {  // 16 digits per load
            const uint4 zz = __ldg(zr + g0 / 8);
            const uint32_t w[4] = {zz.x, zz.y, zz.z, zz.w};
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t word = w[k >> 1] >> (16 * (k & 1));
                const int d0 = (int8_t)(word & 0xFF), d1 = (int8_t)((word >> 8) & 0xFF);
                const uint32_t e = (uint32_t)(d0 + 1) + 3u * (uint32_t)(d1 + 1);  // entry 4 (both zero) is zero
#pragma unroll
                for (int j = 0; j < ZR_TMAX; j++) {
                    if (j >= (int)t) break;
                    const K x = tab[g0 + k][e][j];
                    uint64_t s0 = lo[2 * j] + x.re;
                    hi[2 * j] += s0 < x.re;
                    lo[2 * j] = s0;
                    uint64_t s1 = lo[2 * j + 1] + x.im;
                    hi[2 * j + 1] += s1 < x.im;
                    lo[2 * j + 1] = s1;
                }
            }
        }
    }
    // lo + 2^64 hi (mod q) with 2^64 = 2^32 - 1; hi < 2^16; then into the
    // row's accumulators (a component whose add wraps past 2^64 counts one wrap)
    if (row < R) {
#pragma unroll
        for (int j = 0; j < 2 * ZR_TMAX; j++) {
            if (j >= 2 * (int)t) break;
            const uint64_t c = gl::add(gl::canon(lo[j]), hi[j] * 0xFFFFFFFFull);
            if (c == 0) continue;
            const uint64_t at = (uint64_t)row * 2 * t + j;  // [row][j / 2][re, im]
            const unsigned long long old = atomicAdd(acc_lo + at, (unsigned long long)c);
            if (old + c < old) atomicAdd(acc_wrap + at, 1u);
        }
    }
    __threadfence();
    __syncthreads();
    __shared__ unsigned int s_last;
    if (threadIdx.x == 0) s_last = atomicInc(tickets + blockIdx.x, gridDim.y - 1) == gridDim.y - 1;
    __syncthreads();
    if (!s_last || row >= R) return;
    __threadfence();
    const uint32_t w = row / NEO_D, rho = row % NEO_D;
    for (uint32_t j = 0; j < t; j++) {
        uint64_t c[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const uint64_t at = (uint64_t)row * 2 * t + 2 * j + e;
            // lo + 2^64 wraps (mod q); wraps < 2^32, so wraps (2^32 - 1) < 2^64
            c[e] = gl::add(gl::canon(__ldcg(acc_lo + at)), gl::canon((uint64_t)__ldcg(acc_wrap + at) * 0xFFFFFFFFull));
        }
        y[((uint64_t)w * t + j) * NEO_D + rho] = gl::kmk(c[0], c[1]);
    }
}

// y of R ternary digit rows (layout [w][t][54], row = w * 54 + rho); false
// when the shape does not suit zrows_kernel (the caller keeps its kernel)
int launch_zrows(neo_gpu_ctx* ctx, const int8_t* d_Z, uint32_t R, uint64_t m, uint32_t t, const K* d_v, K* d_y,
                 bool* done) {
    *done = false;
    if (t == 0 || t > ZR_TMAX || m % ZR_CHUNK || R == 0) return NEO_OK;
    const uint32_t groups = (R + ZR_ROWS - 1) / ZR_ROWS;
    const uint64_t chunks = m / ZR_CHUNK;
    // about 8 blocks of 128 rows per SM (latency-bound loop: occupancy hides it)
    uint64_t splits = std::min<uint64_t>(chunks, std::max<uint64_t>(1, (8 * 148 + groups - 1) / groups));
    const uint64_t cps = ((chunks + splits - 1) / splits) * ZR_CHUNK;
    splits = (m + cps - 1) / cps;
    // accumulators [R][t][2] (64-bit sums, then 32-bit wrap counts) and the
    // row groups' tickets, cleared together
    const size_t n_acc = (size_t)R * t * 2;
    const size_t lo_bytes = n_acc * 8, wrap_bytes = n_acc * 4;
    void* scratch = nullptr;
    NEO_CK(ctx, ctx_scratch(ctx, lo_bytes + wrap_bytes + groups * sizeof(unsigned int), &scratch));
    uint8_t* sb = reinterpret_cast<uint8_t*>(scratch);
    NEO_CK(ctx, cudaMemsetAsync(sb, 0, lo_bytes + wrap_bytes + groups * sizeof(unsigned int), ctx->stream));
    zrows_kernel<<<dim3(groups, (uint32_t)splits), ZR_ROWS, 0, ctx->stream>>>(
        d_Z, R, m, t, d_v, cps, reinterpret_cast<unsigned long long*>(sb),
        reinterpret_cast<unsigned int*>(sb + lo_bytes), reinterpret_cast<unsigned int*>(sb + lo_bytes + wrap_bytes), d_y);
    NEO_LAUNCHED(ctx);
    *done = true;
    return NEO_OK;
}

__global__ void y_scalars_kernel(const K* __restrict__ y, uint32_t count, uint32_t b, K* __restrict__ ysc) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;  // (w, j)
    if (q >= count) return;
    K acc = gl::kzero();
    uint64_t pw = 1;
    for (int rho = 0; rho < NEO_D; rho++) {
        acc = gl::kadd(acc, gl::kscale(y[(uint64_t)q * NEO_D + rho], pw));
        pw = gl::mul(pw, b);
    }
    ysc[q] = acc;
}

int launch_me_y(neo_gpu_ctx* ctx, const DevCcs& ccs, const int8_t* d_Z, uint32_t n_w, uint64_t m, const K* d_chi,
                uint32_t ell_n, uint32_t b, K* d_vj, K* d_y, K* d_ysc, bool ternary) {
    uint64_t n_sz = 1ULL << ell_n;
    for (uint32_t j = 0; j < ccs.t; j++) {
        matT_chi_kernel<<<ceil_div(m, 256), 256, 0, ctx->stream>>>(
            ccs.csc_ptr.p + (size_t)j * (m + 1), ccs.csc_row.p + ccs.nnz_off[j], ccs.csc_val.p + ccs.nnz_off[j],
            ccs.is_identity[j], ccs.n, (uint32_t)m, n_sz, d_chi, d_vj + (size_t)j * m);
        NEO_LAUNCHED(ctx);
    }
    bool done = false;
    if (ternary)
        if (int rc = launch_zrows(ctx, d_Z, n_w * NEO_D, m, ccs.t, d_vj, d_y, &done)) return rc;
    if (!done) {
        if (ccs.t <= 4)
            zv_dot_kernel<4><<<n_w * NEO_D, 256, 0, ctx->stream>>>(d_Z, m, ccs.t, d_vj, d_y);
        else
            zv_dot_kernel<16><<<n_w * NEO_D, 256, 0, ctx->stream>>>(d_Z, m, ccs.t, d_vj, d_y);
        NEO_LAUNCHED(ctx);
    }
    if (d_ysc) {
        y_scalars_kernel<<<ceil_div(n_w * ccs.t, 64), 64, 0, ctx->stream>>>(d_y, n_w * ccs.t, b, d_ysc);
        NEO_LAUNCHED(ctx);
    }
    return NEO_OK;
}

static int neo_gpu_me_y_impl_abi(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, const int8_t* Z, uint32_t n_w, uint32_t ell_n,
                            const uint64_t* r, uint32_t b, uint64_t* y, uint64_t* y_scalars) {
    if (!ctx) return NEO_ERR_ARG;
    if (!desc || !Z || !r || !y || !y_scalars || n_w == 0 || ell_n == 0 || ell_n > 30)
        return ctx->fail(NEO_ERR_ARG, "me_y: bad args");
    cudaSetDevice(ctx->device);
    DevCcs ccs;
    int rc = dev_ccs_upload(ctx, desc, ccs);
    if (rc) return rc;
    uint64_t m = desc->m;
    DevBuf<int8_t> dZ;
    DevBuf<K> dr, dchi, dvj, dy, dysc;
    NEO_CK(ctx, dZ.alloc((size_t)n_w * NEO_D * m));
    NEO_CK(ctx, dr.alloc(ell_n));
    NEO_CK(ctx, dchi.alloc(1ULL << ell_n));
    NEO_CK(ctx, dvj.alloc((size_t)ccs.t * m));
    NEO_CK(ctx, dy.alloc((size_t)n_w * ccs.t * NEO_D));
    NEO_CK(ctx, dysc.alloc((size_t)n_w * ccs.t));
    NEO_CK(ctx, cudaMemcpyAsync(dZ.p, Z, dZ.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(dr.p, r, ell_n * 16, cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = launch_chi_table(ctx, dr.p, ell_n, dchi.p))) return rc;
    if ((rc = launch_me_y(ctx, ccs, dZ.p, n_w, m, dchi.p, ell_n, b, dvj.p, dy.p, dysc.p))) return rc;
    NEO_CK(ctx, ctx_d2h(ctx, y, dy.p, dy.bytes()));
    NEO_CK(ctx, ctx_d2h(ctx, y_scalars, dysc.p, dysc.bytes()));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_me_y(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, const int8_t* Z, uint32_t n_w, uint32_t ell_n,
                            const uint64_t* r, uint32_t b, uint64_t* y, uint64_t* y_scalars) { NEO_ABI_GUARD(neo_gpu_me_y_impl_abi(ctx, desc, Z, n_w, ell_n, r, b, y, y_scalars)) }
