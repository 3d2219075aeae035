// commit.cu -- Ajtai commitment c_i = sum_j M[i][j] * z_j in R_q = F_q[X]/Phi_81.
//
// Reference: commit_precomp_ct_row_major (crates/neo-ajtai/src/commit.rs:679-744)
// computes c_i = sum_j rot(a_ij) Z[:, j] column by column.  Here the product
// is taken modulo X^81 - 1 (Phi_81 divides X^81 - 1), i.e. a cyclic
// convolution of length 81 whose matrix entries are the raw PP coefficients,
// and the 81 coefficients are folded back to 54 with X^54 = -X^27 - 1 in the
// epilogue.  This file holds the CUDA-core kernel: split-K over column
// chunks, exact F_q accumulation, then a cross-chunk reduction.
#include "internal.cuh"
#include <algorithm>

using gl::K;

namespace {

constexpr int CHUNK_COLS = 32;    // columns staged per shared-memory tile
constexpr int COMMIT_THREADS = 96;  // >= 81 output coefficients

// partial[(v*n_chunks + chunk)*kappa + i][r], r < 81
__global__ void __launch_bounds__(COMMIT_THREADS)
commit_partial_kernel(const uint64_t* __restrict__ pp, uint32_t kappa, uint64_t m, const int8_t* __restrict__ digits,
                      uint32_t cols_per_block, uint64_t* __restrict__ partial) {
    const uint32_t chunk = blockIdx.x, i = blockIdx.y, v = blockIdx.z;
    const uint32_t n_chunks = gridDim.x;
    __shared__ uint64_t s_a[CHUNK_COLS][NEO_D];
    __shared__ int8_t s_z[CHUNK_COLS][NEO_D + 2];
    const int r = threadIdx.x;
    uint64_t acc = 0;
    const uint64_t j_begin = (uint64_t)chunk * cols_per_block;
    uint64_t j_end = j_begin + cols_per_block;
    if (j_end > m) j_end = m;
    const int8_t* Zv = digits + (uint64_t)v * NEO_D * m;
    for (uint64_t j0 = j_begin; j0 < j_end; j0 += CHUNK_COLS) {
        const int ncol = (int)((j_end - j0) < CHUNK_COLS ? (j_end - j0) : CHUNK_COLS);
        __syncthreads();
        for (int x = threadIdx.x; x < ncol * NEO_D; x += blockDim.x) {
            int c = x / NEO_D, s = x % NEO_D;
            s_a[c][s] = pp[((uint64_t)i * m + j0 + c) * NEO_D + s];
        }
        for (int x = threadIdx.x; x < ncol * NEO_D; x += blockDim.x) {
            int t = x / ncol, c = x % ncol;
            s_z[c][t] = Zv[(uint64_t)t * m + j0 + c];
        }
        __syncthreads();
        if (r < 81) {
            for (int c = 0; c < ncol; c++) {
                // c'[r] += sum_s a[s] * z[(r - s) mod 81], z[p] = 0 for p >= 54
#pragma unroll 6
                for (int s = 0; s < NEO_D; s++) {
                    int p = r - s;
                    p += (p < 0) ? 81 : 0;
                    if (p < NEO_D) {
                        int z = s_z[c][p];
                        if (z == 1) acc = gl::add(acc, s_a[c][s]);
                        else if (z == -1) acc = gl::sub(acc, s_a[c][s]);
                        else if (z != 0) acc = gl::add(acc, gl::mul(s_a[c][s], gl::from_i64(z)));
                    }
                }
            }
        }
    }
    if (r < 81) partial[(((uint64_t)v * n_chunks + chunk) * kappa + i) * 81 + r] = acc;
}

// sum partials over chunks, then fold 81 -> 54: c[r] = c'[r] - c'[r+27] (r>=27) - c'[r+54] (r<27)
__global__ void commit_reduce_kernel(const uint64_t* __restrict__ partial, uint32_t n_chunks, uint32_t kappa,
                                     uint32_t n_vec, uint64_t* __restrict__ out) {
    const uint32_t vi = blockIdx.x;  // v*kappa + i
    const uint32_t v = vi / kappa, i = vi % kappa;
    __shared__ uint64_t s_c[81];
    for (int r = threadIdx.x; r < 81; r += blockDim.x) {
        uint64_t acc = 0;
        for (uint32_t ch = 0; ch < n_chunks; ch++) acc = gl::add(acc, partial[(((uint64_t)v * n_chunks + ch) * kappa + i) * 81 + r]);
        s_c[r] = acc;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < NEO_D; r += blockDim.x) {
        uint64_t c = s_c[r];
        c = gl::sub(c, r >= 27 ? s_c[r + 27] : s_c[r + 54]);
        out[((uint64_t)v * kappa + i) * NEO_D + r] = c;
    }
}

}  // namespace

// PP registry: one entry per (device, m), shared by all contexts
#include <map>
#include <mutex>
static std::mutex g_pp_mu;
static std::map<std::pair<int, uint64_t>, PPEntry*> g_pp;

PPEntry* pp_lookup(int device, uint64_t m) {
    std::lock_guard<std::mutex> lk(g_pp_mu);
    auto it = g_pp.find({device, m});
    return it == g_pp.end() ? nullptr : it->second;
}

int launch_commit(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m, uint64_t* d_out, int digits) {
    PPEntry* pp = pp_lookup(ctx->device, m);
    if (!pp || !pp->kappa) return ctx->fail(NEO_ERR_ARG, "commit: PP not loaded for this m");
    if (pp->tc) {
        // tensor-core path (commit_tc.cu); scratch for every form the call may take
        uint32_t g, k, kb;
        size_t need = 0;
        if (digits != TC_DIGITS_ANY) need = tc_scratch_bytes(n_vec, m, true, pp->kappa, &g, &k, &kb);
        if (digits != TC_DIGITS_SMALL) need = std::max(need, tc_scratch_bytes(n_vec, m, false, pp->kappa, &g, &k, &kb));
        void* scratch = nullptr;
        NEO_CK(ctx, ctx_scratch(ctx, need, &scratch));
        return launch_commit_tc(ctx, pp, d_digits, n_vec, d_out, (uint8_t*)scratch, ctx->d_err, digits);
    }
    const uint32_t kappa = pp->kappa;
    // pick a chunking that fills the GPU: ~4 blocks per SM in total
    uint32_t target_blocks = 148 * 8;
    uint32_t per = (uint32_t)((uint64_t)kappa * n_vec);
    uint32_t n_chunks = (target_blocks + per - 1) / per;
    uint64_t cols_per_block = (m + n_chunks - 1) / n_chunks;
    if (cols_per_block < CHUNK_COLS) cols_per_block = CHUNK_COLS;
    n_chunks = (uint32_t)((m + cols_per_block - 1) / cols_per_block);
    uint64_t* partial = nullptr;
    NEO_CK(ctx, ctx_scratch(ctx, (size_t)n_vec * n_chunks * kappa * 81 * 8, (void**)&partial));
    dim3 grid(n_chunks, kappa, n_vec);
    commit_partial_kernel<<<grid, COMMIT_THREADS, 0, ctx->stream>>>(pp->d_pp, kappa, m, d_digits,
                                                                     (uint32_t)cols_per_block, partial);
    NEO_LAUNCHED(ctx);
    commit_reduce_kernel<<<n_vec * kappa, 96, 0, ctx->stream>>>(partial, n_chunks, kappa, n_vec, d_out);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}

std::mutex& pp_mutex() { return g_pp_mu; }

// Registry slot for (ctx->device, m) with d_pp sized for kappa (caller holds
// pp_mutex()).  The tensor-core tiles of a previous PP are dropped.
int pp_slot(neo_gpu_ctx* ctx, uint32_t kappa, uint64_t m, PPEntry** out) {
    PPEntry*& slot = g_pp[{ctx->device, m}];
    if (!slot) {
        slot = new PPEntry();
        slot->device = ctx->device;
        slot->m = m;
    }
    PPEntry* pp = slot;
    const size_t n = (size_t)kappa * m * NEO_D;
    if (pp->d_pp && pp->kappa != kappa) { cudaFree(pp->d_pp); pp->d_pp = nullptr; pp->kappa = 0; }
    if (!pp->d_pp) NEO_CK(ctx, cudaMalloc(&pp->d_pp, n * 8));
    pp->tc = false;  // the tiles (kept allocated: their size depends on m only) are rebuilt by pp_finish
    *out = pp;
    return NEO_OK;
}

// After d_pp holds the new PP: record kappa and build the tensor-core layout
// (byte limbs, pre-swizzled tiles) when the shape allows it.
int pp_finish(neo_gpu_ctx* ctx, PPEntry* pp, uint32_t kappa) {
    pp->kappa = kappa;
    if (kappa <= 16 && pp->m % 2 == 0) return tc_pp_prepare(ctx, pp);
    if (pp->d_pp_limbs) { cudaFree(pp->d_pp_limbs); pp->d_pp_limbs = nullptr; }
    return NEO_OK;
}

static int neo_gpu_pp_upload_impl_abi(neo_gpu_ctx* ctx, uint32_t kappa, uint64_t m, const uint64_t* coeffs) {
    if (!ctx) return NEO_ERR_ARG;
    if (!coeffs || kappa == 0 || m == 0 || kappa > 64) return ctx->fail(NEO_ERR_ARG, "pp_upload: bad args");
    cudaSetDevice(ctx->device);
    NEO_CK(ctx, ctx_sync(ctx));
    std::lock_guard<std::mutex> lk(g_pp_mu);  // uploads are serialized; replacing a PP in use races (documented)
    PPEntry* pp = nullptr;
    int rc = pp_slot(ctx, kappa, m, &pp);
    if (rc) return rc;
    NEO_CK(ctx, cudaMemcpy(pp->d_pp, coeffs, (size_t)kappa * m * NEO_D * 8, cudaMemcpyHostToDevice));
    return pp_finish(ctx, pp, kappa);
}
extern "C" int neo_gpu_pp_upload(neo_gpu_ctx* ctx, uint32_t kappa, uint64_t m, const uint64_t* coeffs) { NEO_ABI_GUARD(neo_gpu_pp_upload_impl_abi(ctx, kappa, m, coeffs)) }

static int neo_gpu_pp_download_impl_abi(neo_gpu_ctx* ctx, uint64_t m, uint64_t first, uint64_t count, uint64_t* out) {
    if (!ctx) return NEO_ERR_ARG;
    if ((!out && count) || m == 0) return ctx->fail(NEO_ERR_ARG, "pp_download: bad args");
    cudaSetDevice(ctx->device);
    std::lock_guard<std::mutex> lk(g_pp_mu);
    PPEntry* pp = nullptr;
    auto it = g_pp.find({ctx->device, m});
    if (it != g_pp.end()) pp = it->second;
    if (!pp || !pp->d_pp || !pp->kappa) return ctx->fail(NEO_ERR_ARG, "pp_download: PP not loaded for this m");
    const uint64_t total = (uint64_t)pp->kappa * m * NEO_D;
    if (first > total || count > total - first) return ctx->fail(NEO_ERR_ARG, "pp_download: range outside the PP");
    NEO_CK(ctx, ctx_sync(ctx));
    if (count) NEO_CK(ctx, cudaMemcpy(out, pp->d_pp + first, count * 8, cudaMemcpyDeviceToHost));
    return NEO_OK;
}
extern "C" int neo_gpu_pp_download(neo_gpu_ctx* ctx, uint64_t m, uint64_t first, uint64_t count, uint64_t* out) { NEO_ABI_GUARD(neo_gpu_pp_download_impl_abi(ctx, m, first, count, out)) }

static int neo_gpu_commit_impl_abi(neo_gpu_ctx* ctx, const int8_t* digits, uint32_t n_vec, uint64_t m, uint64_t* out) {
    if (!ctx) return NEO_ERR_ARG;
    if (!digits || !out || n_vec == 0 || m == 0) return ctx->fail(NEO_ERR_ARG, "commit: bad args");
    cudaSetDevice(ctx->device);
    PPEntry* pp = pp_lookup(ctx->device, m);
    if (!pp || !pp->kappa) return ctx->fail(NEO_ERR_ARG, "commit: PP not loaded for this m");
    DevBuf<int8_t> dZ;
    DevBuf<uint64_t> dout;
    NEO_CK(ctx, dZ.alloc((size_t)n_vec * NEO_D * m));
    NEO_CK(ctx, dout.alloc((size_t)n_vec * pp->kappa * NEO_D));
    NEO_CK(ctx, cudaMemcpyAsync(dZ.p, digits, dZ.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    int rc = launch_commit(ctx, dZ.p, n_vec, m, dout.p);
    if (rc) return rc;
    if ((rc = check_device_error(ctx))) return rc;
    NEO_CK(ctx, ctx_d2h(ctx, out, dout.p, dout.bytes()));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_commit(neo_gpu_ctx* ctx, const int8_t* digits, uint32_t n_vec, uint64_t m, uint64_t* out) { NEO_ABI_GUARD(neo_gpu_commit_impl_abi(ctx, digits, n_vec, m, out)) }

static int neo_gpu_commit_device_impl_abi(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m,
                                     uint64_t* d_out) {
    if (!ctx) return NEO_ERR_ARG;
    if (!d_digits || !d_out || n_vec == 0 || m == 0) return ctx->fail(NEO_ERR_ARG, "commit_device: bad args");
    cudaSetDevice(ctx->device);
    return launch_commit(ctx, d_digits, n_vec, m, d_out, TC_DIGITS_ANY);
}
extern "C" int neo_gpu_commit_device(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m,
                                     uint64_t* d_out) { NEO_ABI_GUARD(neo_gpu_commit_device_impl_abi(ctx, d_digits, n_vec, m, d_out)) }

static int neo_gpu_commit_device_ex_impl_abi(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m,
                                             uint64_t* d_out, uint32_t flags) {
    if (!ctx) return NEO_ERR_ARG;
    if (!d_digits || !d_out || n_vec == 0 || m == 0 || (flags & ~(uint32_t)NEO_COMMIT_SMALL_DIGITS))
        return ctx->fail(NEO_ERR_ARG, "commit_device_ex: bad args");
    cudaSetDevice(ctx->device);
    return launch_commit(ctx, d_digits, n_vec, m, d_out,
                         (flags & NEO_COMMIT_SMALL_DIGITS) ? TC_DIGITS_SMALL : TC_DIGITS_ANY);
}
extern "C" int neo_gpu_commit_device_ex(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m,
                                        uint64_t* d_out, uint32_t flags) {
    NEO_ABI_GUARD(neo_gpu_commit_device_ex_impl_abi(ctx, d_digits, n_vec, m, d_out, flags))
}

// ---------------------------------------------------------------------------
// Allocation-free commitment.
//
// Some callers cannot allocate device memory at the moment they commit: code
// running while a CUDA stream is being captured into a graph (cudaMalloc and
// cudaFree are not stream-ordered and break or serialize the capture), hosts
// whose framework owns every device byte through its own pool and forbids
// untracked allocations, and latency-critical provers for which the implicit
// device synchronization of cudaMalloc/cudaFree would stall other streams.
// For them, neo_gpu_commit_noalloc runs the CUDA-core commitment kernels above
// with their split-K partial sums in the fixed device array below instead of
// context scratch.  The array is part of the library image, so every GPU that
// loads the library holds its 4 MiB until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {
constexpr uint64_t NOALLOC_SCRATCH_WORDS = 1ull << 19;  // 524288 uint64 = 4 MiB of partial sums
static __device__ __align__(256) uint64_t g_commit_noalloc_scratch[NOALLOC_SCRATCH_WORDS];
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
uint64_t* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};
}  // namespace

static int neo_gpu_commit_noalloc_impl_abi(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m,
                                      uint64_t* d_out) {
    if (!ctx) return NEO_ERR_ARG;
    if (!d_digits || !d_out || n_vec == 0 || m == 0) return ctx->fail(NEO_ERR_ARG, "commit_noalloc: bad args");
    PPEntry* pp = pp_lookup(ctx->device, m);
    // kappa and the coefficient pointer are read once: a PP being generated or
    // re-uploaded, or one whose generation failed, has kappa = 0 (no usable PP)
    const uint32_t kappa = pp ? pp->kappa : 0;
    const uint64_t* d_pp = pp ? pp->d_pp : nullptr;
    if (!kappa || !d_pp) return ctx->fail(NEO_ERR_ARG, "commit_noalloc: PP not loaded for this m");
    if (ctx->device < 0 || ctx->device >= NOALLOC_MAX_DEVICES) return ctx->fail(NEO_ERR_UNSUPPORTED, "commit_noalloc: device index");
    const uint64_t per_chunk = (uint64_t)n_vec * kappa * 81;  // partial words needed per column chunk
    if (per_chunk > NOALLOC_SCRATCH_WORDS)
        return ctx->fail(NEO_ERR_ARG,
                         "commit_noalloc: n_vec * kappa * 81 exceeds the fixed 524288-word scratch "
                         "(at most 404 vectors for kappa = 16); use neo_gpu_commit_device");
    NEO_CK(ctx, cudaSetDevice(ctx->device));
    // one-time set-up on this device: the array's device address (the host-side
    // symbol is only a stand-in and must never be handed to a kernel)
    uint64_t* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[ctx->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_commit_noalloc_scratch);
            if (e != cudaSuccess || !p) return ctx->fail(NEO_ERR_CUDA, "commit_noalloc: cudaGetSymbolAddress", e);
            g_noalloc_ptr[ctx->device] = static_cast<uint64_t*>(p);
        }
        scratch = g_noalloc_ptr[ctx->device];
    }
    // same chunking rule as launch_commit: about 1184 blocks in all, so
    // n_chunks * kappa * n_vec stays near 1184 and, with 81 partial words per
    // (chunk, row, vector), far inside the scratch once per_chunk fits
    uint32_t target_blocks = 148 * 8;
    uint32_t per = (uint32_t)((uint64_t)kappa * n_vec);
    uint64_t n_chunks = (target_blocks + per - 1) / per;
    uint64_t cols_per_block = (m + n_chunks - 1) / n_chunks;
    if (cols_per_block < CHUNK_COLS) cols_per_block = CHUNK_COLS;
    n_chunks = (m + cols_per_block - 1) / cols_per_block;
    if (n_chunks * per_chunk > NOALLOC_SCRATCH_WORDS)
        return ctx->fail(NEO_ERR_INVARIANT, "commit_noalloc: partial sums exceed the fixed scratch");
    dim3 grid((uint32_t)n_chunks, kappa, n_vec);
    // every partial word a reduce reads is written by commit_partial_kernel first,
    // so the array needs no clearing between calls
    commit_partial_kernel<<<grid, COMMIT_THREADS, 0, ctx->stream>>>(d_pp, kappa, m, d_digits,
                                                                     (uint32_t)cols_per_block, scratch);
    NEO_LAUNCHED(ctx);
    commit_reduce_kernel<<<n_vec * kappa, 96, 0, ctx->stream>>>(scratch, (uint32_t)n_chunks, kappa, n_vec, d_out);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}
extern "C" int neo_gpu_commit_noalloc(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m,
                                      uint64_t* d_out) { NEO_ABI_GUARD(neo_gpu_commit_noalloc_impl_abi(ctx, d_digits, n_vec, m, d_out)) }
