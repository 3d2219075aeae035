// internal.cuh -- context, status handling and device buffers shared by the
// CUDA translation units of libneo_gpu.so.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/neo_gpu.h"
#include "abi_guard.h"
#include "gl.cuh"

#define NEO_D 54
// bytes per rot(a) row in the RLC mix scratch: 54 int8 entries, zero padded
constexpr int RLC_ROT_ROW = 64;

struct neo_gpu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t launches = 0;
    uint32_t* d_err = nullptr;       // device error word (bounded-wait timeouts); 0 = ok
    void* scratch = nullptr;         // growable per-context scratch (stream-ordered use)
    size_t scratch_bytes = 0;
    // the last chi table a memory oracle built (the time-lane oracles of a
    // step share their point): key = ell then the point's words
    void* chi_cache = nullptr;
    size_t chi_cache_bytes = 0;
    std::vector<uint64_t> chi_key;
    int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
        char buf[512];
        if (e != cudaSuccess)
            snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
        else
            snprintf(buf, sizeof buf, "%s", what);
        err = buf;
        return code;
    }
};

// wait for the context's stream (a spinning stream synchronization: batch
// workers that slept in blocking waits were measured no faster)
inline cudaError_t ctx_sync(neo_gpu_ctx* c) { return cudaStreamSynchronize(c->stream); }

// device -> host copy on the context's stream
inline cudaError_t ctx_d2h(neo_gpu_ctx* c, void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
}

#define NEO_CK(ctx, call)                                                         \
    do {                                                                          \
        cudaError_t _e = (call);                                                  \
        if (_e != cudaSuccess) {                                                  \
            return (ctx)->fail(_e == cudaErrorMemoryAllocation ? NEO_ERR_OOM      \
                                                               : NEO_ERR_CUDA,    \
                               #call, _e);                                        \
        }                                                                         \
    } while (0)

#define NEO_LAUNCHED(ctx)                                                         \
    do {                                                                          \
        (ctx)->launches++;                                                        \
        cudaError_t _e = cudaGetLastError();                                      \
        if (_e != cudaSuccess) return (ctx)->fail(NEO_ERR_CUDA, "kernel launch", _e); \
    } while (0)

// Ajtai public parameters of one m on one device, shared by every context on
// that device (the reference keeps one PP per (d, m) in a global registry,
// crates/neo-ajtai/src/s_module.rs:23-222).
struct PPEntry {
    int device = 0;
    uint64_t m = 0;
    uint32_t kappa = 0;
    uint64_t* d_pp = nullptr;       // [kappa][m][54] canonical u64
    uint8_t* d_pp_limbs = nullptr;  // tensor-core tiles: [m/2][128 rows][128 B], pre-swizzled
    bool tc = false;                // d_pp_limbs holds the tiles of the current d_pp
};
PPEntry* pp_lookup(int device, uint64_t m);
// PP registry writes (commit.cu): pp_slot / pp_finish are called with pp_mutex() held
#include <mutex>
std::mutex& pp_mutex();
int pp_slot(neo_gpu_ctx* ctx, uint32_t kappa, uint64_t m, PPEntry** out);
int pp_finish(neo_gpu_ctx* ctx, PPEntry* pp, uint32_t kappa);

// Owning device buffer (freed on scope exit).
// Stream of this thread's stream-ordered allocations (set by batch workers,
// whose thread uses a single context); null: plain cudaMalloc / cudaFree.
extern thread_local cudaStream_t g_alloc_stream;

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;  // stream the allocation was ordered on (null: cudaMalloc)
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    size_t cap = 0;
    cudaError_t alloc(size_t count) {
        release();
        n = count;
        cap = count;
        if (count == 0) return cudaSuccess;
        s = g_alloc_stream;
        if (s) return cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), s);
        return cudaMalloc(&p, count * sizeof(T));
    }
    // keep the allocation when it is large enough (reused workspaces)
    cudaError_t ensure(size_t count) {
        if (p && count <= cap) {
            n = count;
            return cudaSuccess;
        }
        return alloc(count);
    }
    void release() {
        if (p) {
            if (s) cudaFreeAsync(p, s);
            else cudaFree(p);
        }
        p = nullptr;
        s = nullptr;
        n = 0;
        cap = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// Page-locked host buffer: a cudaMemcpyAsync from or to it is queued on the
// stream and does not wait for the stream's earlier work (a pageable source
// makes the copy synchronous).  Reused across rounds; freed on scope exit.
template <typename T>
struct HostBuf {
    T* p = nullptr;
    size_t cap = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() {
        if (p) cudaFreeHost(p);
    }
    cudaError_t ensure(size_t count) {
        if (p && count <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&p), (count ? count : 1) * sizeof(T), cudaHostAllocDefault);
        if (e == cudaSuccess) cap = count;
        return e;
    }
};

// Device-side CCS copy in both CSR (row SpMV) and CSC (transposed SpMV) form.
struct DevCcs {
    uint32_t n = 0, m = 0, t = 0;
    std::vector<uint8_t> is_identity;
    std::vector<uint64_t> f_coeff;
    std::vector<uint32_t> f_exps;
    uint32_t n_terms = 0;
    // per matrix offsets into the packed arrays
    std::vector<uint64_t> nnz_off;
    DevBuf<uint64_t> csr_ptr;   // [t][n+1] (relative to nnz_off[j])
    DevBuf<uint32_t> csr_col;   // [nnz]
    DevBuf<uint64_t> csr_val;   // [nnz]
    DevBuf<uint64_t> csc_ptr;   // [t][m+1]
    DevBuf<uint32_t> csc_row;   // [nnz]
    DevBuf<uint64_t> csc_val;   // [nnz]
};
// Grow-only scratch owned by the context; valid until the next call that grows it.
inline cudaError_t ctx_scratch(neo_gpu_ctx* ctx, size_t bytes, void** p) {
    if (bytes > ctx->scratch_bytes) {
        const bool pooled = g_alloc_stream == ctx->stream;  // stream-ordered: no device-wide wait
        if (ctx->scratch) {
            if (pooled) {
                cudaFreeAsync(ctx->scratch, ctx->stream);
            } else {
                cudaStreamSynchronize(ctx->stream);
                cudaFree(ctx->scratch);
            }
            ctx->scratch = nullptr;
            ctx->scratch_bytes = 0;
        }
        cudaError_t e = pooled ? cudaMallocAsync(&ctx->scratch, bytes, ctx->stream) : cudaMalloc(&ctx->scratch, bytes);
        if (e != cudaSuccess) return e;
        ctx->scratch_bytes = bytes;
    }
    *p = ctx->scratch;
    return cudaSuccess;
}
int dev_ccs_upload(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, DevCcs& out);

// Kernels callable from several translation units.
int launch_chi_table(neo_gpu_ctx* ctx, const gl::K* d_bits, uint32_t nbits, gl::K* d_out);
// chi(bits[j+1..nbits)) for every j < nbits, table j at 2^nbits - 2^(nbits-j), in one launch
int launch_suffix_chi_tables(neo_gpu_ctx* ctx, const gl::K* d_bits, uint32_t nbits, gl::K* d_out);
int launch_me_y(neo_gpu_ctx* ctx, const DevCcs& ccs, const int8_t* d_Z, uint32_t n_w, uint64_t m,
                const gl::K* d_chi, uint32_t ell_n, uint32_t b, gl::K* d_vj_scratch, gl::K* d_y,
                gl::K* d_ysc, bool ternary = false);
// y[row][j] = sum_c Z[row][c] v[j][c] of R ternary digit rows (y layout [w][t][54]); *done = false
// (nothing launched) when m % 64 != 0 or t > 4
int launch_zrows(neo_gpu_ctx* ctx, const int8_t* d_Z, uint32_t R, uint64_t m, uint32_t t, const gl::K* d_v,
                 gl::K* d_y, bool* done);
// What the caller knows about the digits of a commitment: any int8
// (TC_DIGITS_ANY: the cyclic tensor-core form), |digit| <= 63 by construction
// (TC_DIGITS_SMALL: the small-digit form, a violation is reported through the
// device error word), or nothing (TC_DIGITS_CHECK: the small-digit form after
// one device check, else the cyclic form).
enum { TC_DIGITS_ANY = 0, TC_DIGITS_SMALL = 1, TC_DIGITS_CHECK = 2 };
int launch_commit(neo_gpu_ctx* ctx, const int8_t* d_digits, uint32_t n_vec, uint64_t m, uint64_t* d_out,
                  int digits = TC_DIGITS_CHECK);
int tc_pp_prepare(neo_gpu_ctx* ctx, PPEntry* pp);
size_t tc_scratch_bytes(uint32_t n_vec, uint64_t m, bool small, uint32_t kappa, uint32_t* n_groups,
                        uint32_t* n_ksplit, uint32_t* kb_per_cta);
int launch_commit_tc(neo_gpu_ctx* ctx, const PPEntry* pp, const int8_t* d_digits, uint32_t n_vec, uint64_t* d_out,
                     uint8_t* scratch, uint32_t* d_err, int digits);
// reads and clears the device error word (synchronizes the stream)
int check_device_error(neo_gpu_ctx* ctx);

// AddressLookupOracle weight table and claimed sum from device columns (mem_oracle.cu);
// ws (may be null) keeps the temporaries across calls
struct AddrWs {
    DevBuf<gl::K> chi, part, out1;
    DevBuf<unsigned long long> acc;
};
int addr_weights_device(neo_gpu_ctx* ctx, uint32_t ell, const gl::K* d_rcycle, uint32_t A, const gl::K* d_has,
                        const gl::K* d_bits, const gl::K* d_table, uint64_t table_len, gl::K* d_w, gl::K* claim,
                        AddrWs* ws);
// Memory-oracle builds that reuse the object in *slot (mem_oracle.cu)
int mem_oracle_build_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point, uint32_t ell_addr,
                            const uint64_t* r_addr, const uint64_t* init_at_r_addr, uint32_t n_cols,
                            const uint64_t* d_cols, const uint64_t* weights, uint64_t* claim,
                            neo_gpu_mem_oracle** slot);
int twist_addr_build_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle, uint32_t ell_addr,
                            uint64_t n_init, const uint64_t* init_addr, const uint64_t* init_val,
                            const uint64_t* d_cols, neo_gpu_twist_addr** slot);

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

// A kernel's dynamic shared-memory limit (cudaFuncAttributeMaxDynamicSharedMemorySize)
// is a process-wide attribute of the function.  Host threads that set it to
// their own launch's size would undo each other: a thread launching with 56 KB
// fails ("too many resources requested for launch") when another thread set
// 4 KB in between.  SmemLimit only ever raises the attribute, under a lock, so
// every launch that follows its own at_least() call stays within the limit.
struct SmemLimit {
    std::mutex mu;
    size_t cur = 48 * 1024;
    template <typename Kernel>
    cudaError_t at_least(Kernel* kernel, size_t bytes) {
        std::lock_guard<std::mutex> lk(mu);
        if (bytes > cur) cur = bytes;
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cur);
    }
};
