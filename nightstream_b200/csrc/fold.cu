// fold.cu -- device-resident Neo fold step for one shard, with the optional
// shared-CPU-bus memory sidecar (Twist read/write memories, Shout lookups):
// MCS commit -> [Shout / Twist address pre-time sum-checks] -> Pi_CCS
// (batched time rounds over the CCS and Route-A memory claims + Ajtai rounds)
// -> ME outputs (+ bus openings) -> [Twist val-eval batch, val-lane CPU ME
// claims] -> Pi_RLC -> Pi_DEC (main lane, 12 child commitments) -> [val lane
// RLC / DEC].
//
// Reference: fold_shard_prove_impl (crates/neo-fold/src/shard.rs:1725-2283),
// prove_rlc_dec_lane (shard.rs:1170-1331), prove_route_a_batched_time
// (crates/neo-fold/src/memory_sidecar/route_a_time.rs:28-152), the memory
// sidecar (memory_sidecar/memory.rs:86-1670, cpu_bus.rs:195-320, 969-1016,
// transcript.rs:4-63, utils.rs:43-71), the sum-check drivers
// (crates/neo-reductions/src/sumcheck.rs:124-456) and their domain separation
// (memory_sidecar/sumcheck_ds.rs:11-77).  The transcript calls are issued in
// the reference's order with the reference's labels.
//
// All witness digit planes live in one device buffer Zall[1 + k_rho][54][m]:
// slot 0 holds the step's MCS witness, slots 1..k_rho the carried children.
// Pi_DEC writes the new children straight into slots 1..k_rho.  Bus columns
// (the tail of z: cell (col, j) at bus_base + col * steps + j, time row
// m_in + j) are decoded into dense K time columns d_cols[bus_cols][2^ell_n].
#include <future>
#include <nvtx3/nvToolsExt.h>
#include "internal.cuh"

#include <list>
#include <mutex>
#include "transcript.h"
#include <algorithm>
#include <chrono>
#include <memory>
#include <string>

using gl::K;

int rlc_mix_device(neo_gpu_ctx* ctx, const int8_t* rho_coeffs_host, const int8_t* d_Zs, uint32_t count, uint64_t m,
                   int32_t* d_Zmix, int8_t* d_rot_scratch);
int split_b_device(neo_gpu_ctx* ctx, const int32_t* d_Zmix, uint64_t len, uint32_t k, uint32_t b, int8_t* d_planes,
                   uint32_t* d_flags);
__global__ void decomp_b2_kernel(const uint64_t* __restrict__ z, uint64_t m, int8_t* __restrict__ Z);

namespace {

struct MeInst {
    std::vector<uint64_t> c;      // kappa*54 (Commitment.data, column-major)
    std::vector<uint64_t> X;      // 54*m_in row-major
    std::vector<K> r;             // ell_n
    std::vector<K> y;             // (t + bus_cols) * 2^ell_d (padded)
    std::vector<K> ysc;           // t + bus_cols
    uint32_t m_in = 0;
    uint8_t digest[32] = {0};
};

struct ShoutInst {
    uint32_t ea = 0;                      // ell_addr = d * ell
    uint64_t k = 0, d = 0, n_side = 0, ell = 0;
    std::vector<uint64_t> table;          // F_q entries
    uint8_t digest[32] = {0};
    DevBuf<K> d_table;                    // min(len, 2^ea) entries as K, zero padded to 2^ea
    uint32_t col0 = 0;                    // addr bits col0.., has_lookup col0+ea, val col0+ea+1
};

struct TwistInst {
    uint32_t ea = 0;
    uint64_t k = 0, d = 0, n_side = 0, ell = 0;
    std::vector<uint64_t> init_addr, init_val;  // MemInit::Sparse (empty: MemInit::Zero)
    uint8_t digest[32] = {0};
    uint32_t col0 = 0;  // ra col0.., wa col0+ea.., has_read +2ea, has_write +2ea+1, wv +2, rv +3, inc +4
    // trace steps (neo_gpu_shard_fold_step_trace): the memory, dense over
    // 2^ea cells in device memory, at the start of the next chunk
    DevBuf<uint64_t> d_state;
    bool state_valid = false;
};

static std::vector<uint8_t> le64(uint64_t v) {
    std::vector<uint8_t> b(8);
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * i));
    return b;
}

// out[v][r] = sum_i rot_i[r][k] * V_i[v][k]  over F_q, element stride `stride`
// (Commitment mixing mix_rhos_commits and S-action on y vectors, common.rs:398-430).
// rot rows are RLC_ROT_ROW bytes apart (the RLC mix scratch).  A block
// (64 x 16 threads) owns one output vector: thread (r, i) forms
// sum_k rot_i[r][k] V_i[v][k] for 16 inputs at a time.  rot entries are small
// integers, so the terms are summed exactly in 128 bits (positive and negative
// coefficients apart) and reduced once; the per-input partials are then
// added mod q in shared memory.
__global__ void __launch_bounds__(1024) rot_mix_kernel(const int8_t* __restrict__ rot, uint32_t count,
                                                       const uint64_t* __restrict__ V, uint32_t nv, uint32_t stride,
                                                       uint64_t* __restrict__ out) {
    __shared__ uint64_t xs[16][NEO_D];
    __shared__ uint64_t part[16][NEO_D];
    const uint32_t v = blockIdx.x / stride, comp = blockIdx.x % stride;
    const int r = threadIdx.x, ii = threadIdx.y;
    const bool row = r < NEO_D;
    uint64_t total = 0;
    for (uint32_t i0 = 0; i0 < count; i0 += 16) {
        const uint32_t i = i0 + ii;
        const bool live = row && i < count;
        if (live) xs[ii][r] = V[(((size_t)i * nv + v) * NEO_D + r) * stride + comp];
        __syncthreads();
        if (live) {
            const int4* R4 = reinterpret_cast<const int4*>(rot + ((size_t)i * NEO_D + r) * RLC_ROT_ROW);
            const int4 q[4] = {R4[0], R4[1], R4[2], R4[3]};
            uint64_t pl = 0, ph = 0, nl = 0, nh = 0;  // < 54 * 4 * 2^64 < 2^72 each
#pragma unroll
            for (int k = 0; k < NEO_D; k++) {
                const int4& w4 = q[k >> 4];
                const int w = ((k >> 2) & 3) == 0 ? w4.x : ((k >> 2) & 3) == 1 ? w4.y : ((k >> 2) & 3) == 2 ? w4.z : w4.w;
                const int c = (int)(int8_t)(w >> (8 * (k & 3)));
                const uint64_t x = xs[ii][k];
                const uint64_t a = (uint64_t)(c < 0 ? -c : c);
                const uint64_t lo = x * a, hi = __umul64hi(x, a);
                if (c > 0) {
                    pl += lo;
                    ph += hi + (pl < lo);
                } else if (c < 0) {
                    nl += lo;
                    nh += hi + (nl < lo);
                }
            }
            part[ii][r] = gl::sub(gl::reduce128(pl, ph), gl::reduce128(nl, nh));
        } else if (row) {
            part[ii][r] = 0;
        }
        __syncthreads();
        if (ii == 0 && row)
            for (int j = 0; j < 16; j++) total = gl::add(total, part[j][r]);
        __syncthreads();
    }
    if (ii == 0 && row) out[((size_t)v * NEO_D + r) * stride + comp] = total;
}

// child ME claims: y[w][j][rho] = sum_c P_w[rho][c] v_j[c] (zv_dot in core.cu uses the same math)
__global__ void __launch_bounds__(256) child_y_kernel(const int8_t* __restrict__ Z, uint64_t m, uint32_t t,
                                                      const K* __restrict__ v, K* __restrict__ y) {
    const uint32_t row = blockIdx.x;
    const int8_t* zr = Z + (uint64_t)row * m;
    K acc[4] = {gl::kzero(), gl::kzero(), gl::kzero(), gl::kzero()};
    for (uint64_t c = threadIdx.x; c < m; c += blockDim.x) {
        int z = zr[c];
        if (z == 0) continue;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (j < (int)t) {
                K x = v[(uint64_t)j * m + c];
                acc[j] = z == 1 ? gl::kadd(acc[j], x) : (z == -1 ? gl::ksub(acc[j], x) : gl::kadd(acc[j], gl::kscale_small(x, z)));
            }
    }
    __shared__ K red[4][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 4; j++) {
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
        for (int w = 0; w < 8; w++) a = gl::kadd(a, red[threadIdx.x][w]);
        uint32_t wi = row / NEO_D, rho = row % NEO_D;
        y[((uint64_t)wi * t + threadIdx.x) * NEO_D + rho] = a;
    }
}

// build_time_sparse_from_bus_col (memory_sidecar/cpu_bus.rs:976-1016), dense:
// out[c][t] = z[bus_base + c*steps + (t - m_in)] for m_in <= t < m_in + steps, else 0
__global__ void bus_decode_kernel(const uint64_t* __restrict__ z, uint32_t m_in, uint64_t bus_base, uint64_t steps,
                                  uint32_t ncols, uint64_t L, K* __restrict__ out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= (uint64_t)ncols * L) return;
    const uint64_t c = i / L, t = i - c * L;
    K v = gl::kzero();
    if (t >= m_in && t - m_in < steps) v = gl::kfq(gl::canon(z[bus_base + c * steps + (t - m_in)]));
    out[i] = v;
}

// χ_r(m_in + j) for the bus time rows (cpu_bus.rs:180-192, 279-283)
__global__ void bus_weights_kernel(const K* __restrict__ r, uint32_t ell, uint32_t m_in, uint64_t steps,
                                   K* __restrict__ w) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j >= steps) return;
    const uint64_t row = m_in + j;
    K acc = gl::kone();
    for (uint32_t b = 0; b < ell; b++) acc = gl::kmul(acc, ((row >> b) & 1) ? r[b] : gl::ksub(gl::kone(), r[b]));
    w[j] = acc;
}

// bus openings y[w][c][rho] = Σ_j χ_r(m_in + j) Z_w[rho][bus_base + c*steps + j]
// (append_bus_openings_to_me_instance, cpu_bus.rs:195-320); block per (c, rho), grid.y witnesses
// One warp per (witness, bus column, digit row): y = sum_j Z[row][bus_base +
// c steps + j] w[j] over the chunk's steps (lanes stride the steps; the
// weights are shared by every item and stay in L1/L2), a warp reduction, no
// block barrier.  items = n_w * ncols * 54.
constexpr int BUS_OPEN_WARPS = 8;
__global__ void __launch_bounds__(32 * BUS_OPEN_WARPS) bus_open_kernel(const int8_t* __restrict__ Z, uint64_t m,
                                                                      uint64_t bus_base, uint64_t steps, uint32_t ncols,
                                                                      uint64_t items, const K* __restrict__ w,
                                                                      K* __restrict__ y) {
    const uint64_t item = (uint64_t)blockIdx.x * BUS_OPEN_WARPS + (threadIdx.x >> 5);
    if (item >= items) return;  // warp-uniform
    const int lane = threadIdx.x & 31;
    const uint32_t rho = (uint32_t)(item % NEO_D);
    const uint32_t c = (uint32_t)((item / NEO_D) % ncols);
    const uint64_t wi = item / ((uint64_t)NEO_D * ncols);
    const int8_t* zr = Z + (wi * NEO_D + rho) * m + bus_base + (uint64_t)c * steps;
    K acc = gl::kzero();
    for (uint64_t j = lane; j < steps; j += 32) {
        const int z = zr[j];
        if (z == 1) acc = gl::kadd(acc, w[j]);
        else if (z == -1) acc = gl::ksub(acc, w[j]);
        else if (z != 0) acc = gl::kadd(acc, gl::kscale_small(w[j], z));
    }
    for (int o = 16; o > 0; o >>= 1) {
        K b;
        b.re = __shfl_xor_sync(0xffffffffu, acc.re, o);
        b.im = __shfl_xor_sync(0xffffffffu, acc.im, o);
        acc = gl::kadd(acc, b);
    }
    if (lane == 0) y[(wi * ncols + c) * NEO_D + rho] = acc;
}

}  // namespace

// ---------------------------------------------------------------------------
// The last fold step in the field order of the reference's StepProof
// (crates/neo-fold/src/shard_proof_types.rs:45-131): the pieces the
// transcript-order proof dump interleaves, kept for neo_gpu_shard_step_proof.
struct BatchRec {  // one batched sum-check (BatchedTimeProof-like)
    std::vector<std::string> labels;
    std::vector<uint32_t> degs;
    std::vector<K> sums;
    std::vector<std::vector<std::vector<K>>> polys;  // [claim][round][coefficient]
    std::vector<K> chals, finals;
};
struct LaneRec {  // RlcDecProof
    bool present = false;
    std::vector<int8_t> rhos;  // [k][54] coefficients of rho_i = rot(a_i)
    MeInst parent;
    std::vector<MeInst> children;
};
struct StepRecord {
    bool valid = false;
    std::vector<MeInst> ccs_out;
    std::vector<std::vector<K>> ajtai_polys;  // PiCcsProof::sumcheck_rounds (the Ajtai rounds)
    std::vector<K> ajtai_chals;
    K T{}, final_sum{};
    std::vector<K> alpha, beta_a, beta_r;
    K gamma{};
    LaneRec main, val;
    BatchRec time;
    std::vector<MeInst> cpu_me_val;
    bool has_shout = false;
    std::vector<K> shout_sums;
    uint64_t shout_active = 0;
    BatchRec shout_pre;
    std::vector<BatchRec> twist_pre;
    uint32_t n_lut = 0;
    bool has_val_eval = false, val_has_prev = false;
    BatchRec val_eval;
};

struct neo_gpu_shard {
    neo_gpu_ctx* ctx = nullptr;
    DevCcs ccs;
    // batched sum-check rounds: every claim's round values in one device array,
    // read back with one copy per round (page-locked), and the partial sums of
    // the multi-claim memory kernels
    DevBuf<K> d_round, d_mpart;
    HostBuf<K> h_round;
    DevBuf<uint64_t> d_events;  // a trace chunk's packed events (neo_gpu_shard_fold_step_trace)
    HostBuf<uint64_t> h_events;
    StepRecord rec;  // the last step, for neo_gpu_shard_step_proof
    uint32_t kappa = 16;
    uint32_t n = 0, m32 = 0, t = 0, ell_n = 0, ell_d = 6, d_sc = 6, k_rho = 12, b = 2, m_in = 1, lambda = 127;
    uint64_t m = 0;
    int64_t slack_bits = 0;
    uint64_t mat_digest[4] = {0, 0, 0, 0};
    std::unique_ptr<neo::Transcript> tr;
    uint32_t step_idx = 0;
    DevBuf<int8_t> Zall;
    std::vector<MeInst> acc;
    DevBuf<uint64_t> d_z, d_commits, d_mixv, d_mixo;
    DevBuf<int32_t> d_mix;
    DevBuf<int8_t> d_rot;
    DevBuf<uint32_t> d_flags;
    DevBuf<K> d_ychild;
    neo_gpu_ccs_oracle* orc = nullptr;  // Pi_CCS oracle workspace reused across steps
    std::vector<uint64_t> proof;  // canonical dump of the last step
    double stats[12] = {0};       // host ms per phase of the last step, see neo_gpu_shard_step_stats
    // ---- shared CPU bus (memory sidecar) ----
    uint64_t steps = 0, bus_base = 0;
    uint32_t bus_cols = 0;
    std::vector<std::unique_ptr<ShoutInst>> shout;
    std::vector<std::unique_ptr<TwistInst>> twist;
    DevBuf<K> d_cols, d_prev_cols, d_asm, d_busw, d_busy, d_r, d_chi, d_vj, d_yv, d_yvsc, d_w;
    DevBuf<int8_t> valwit;     // [2][54][m]: this step's and the previous step's MCS digits
    DevBuf<int8_t> valplanes;  // [k_rho][54][m]: val-lane DEC children
    bool has_prev = false;
    std::vector<uint64_t> prev_c, prev_X;
    uint64_t val_obligations = 0;
    std::vector<neo_gpu_mem_oracle*> mem_slots;  // memory oracles, rebuilt in place every step
    std::vector<neo_gpu_twist_addr*> ta_slots;
    AddrWs addr_ws;
};

using hclock = std::chrono::steady_clock;
static inline double ms_since(hclock::time_point t0) {
    return std::chrono::duration<double, std::milli>(hclock::now() - t0).count();
}

// NVTX ranges name a fold step and its phases (witness, bind, ccs_build,
// time_rounds, ajtai_rounds, me_outputs, rlc_dec, val_lane) in the NVTX domain
// "neo", for profilers: nsys timelines, ncu --nvtx --nvtx-include
// "neo@fold_step/rlc_dec/".  With no tool attached a push or pop is one call
// that returns.  Ranges still open when the step returns (an error path) are
// closed here, so the thread's range stack stays balanced.
namespace {
nvtxDomainHandle_t nvtx_domain() {
    static nvtxDomainHandle_t d = nvtxDomainCreateA("neo");
    return d;
}
struct NvtxStep {
    int depth = 0;
    void push(const char* name) {
        nvtxEventAttributes_t a = {};
        a.version = NVTX_VERSION;
        a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
        a.messageType = NVTX_MESSAGE_TYPE_ASCII;
        a.message.ascii = name;
        nvtxDomainRangePushEx(nvtx_domain(), &a);
        depth++;
    }
    void next(const char* name) {
        pop();
        push(name);
    }
    void pop() {
        if (depth) {
            nvtxDomainRangePop(nvtx_domain());
            depth--;
        }
    }
    ~NvtxStep() {
        while (depth) pop();
    }
};
}  // namespace

static void header_params(neo_gpu_shard* sh) {
    // goldilocks_auto_r1cs_ccs (crates/neo-params/src/lib.rs:181-222) with
    // extension_check (lib.rs:246-304): largest lambda <= 127 (>= 96) whose
    // s = 2 slack is >= 2 bits.
    const unsigned __int128 q = (unsigned __int128)GL_Q;
    const unsigned __int128 q2 = q * q;
    const uint32_t ell = sh->ell_n + sh->ell_d;
    auto bitlen = [](unsigned __int128 x) {
        int b = 0;
        while (x) { b++; x >>= 1; }
        return b;
    };
    const unsigned __int128 ld = (unsigned __int128)ell * sh->d_sc;
    const unsigned __int128 U128_MAX = ~(unsigned __int128)0;
    for (uint32_t lam = 127; lam >= 96; lam--) {
        // rhs = 2^lam * ell * d_sc; an overflow means s = 2 is unsupported (checked_shl/checked_mul)
        unsigned __int128 p2 = (unsigned __int128)1 << lam;
        if (ld != 0 && p2 > U128_MAX / ld) continue;
        unsigned __int128 rhs = p2 * ld;
        if (q2 < rhs) continue;
        int slack = bitlen(q2) - bitlen(rhs);
        // rhs.checked_shl(slack): shift only when the result stays below 2^128
        if (slack < 128 && bitlen(rhs) + slack <= 128 && q2 < (rhs << slack)) slack -= 1;
        if (slack >= 2) {
            sh->lambda = lam;
            sh->slack_bits = slack;
            return;
        }
    }
}

// digest_ccs_matrices (crates/neo-reductions/src/engines/utils.rs:214-321)
// The matrix digest is a sequential width-16 sponge over every nonzero
// (O(nnz) permutations, 0.17 s at n = 2^16), computed once per CCS: the
// reference keeps it in ShardProverContext (shard.rs:2557-2560).  Shards
// created for a CCS seen before (the same circuit proving many shards) reuse
// it; entries are matched on an exact copy of the matrix data, least recently
// used first out, at most 512 MiB of copies.
namespace {
struct DigestEntry {
    uint32_t n = 0, m = 0, t = 0;
    std::vector<uint8_t> ident;
    std::vector<uint64_t> col_ptr, nnz_off, vals;
    std::vector<uint32_t> row_idx;
    uint64_t out[4] = {0, 0, 0, 0};
    size_t bytes() const {
        return ident.size() + 8 * (col_ptr.size() + nnz_off.size() + vals.size()) + 4 * row_idx.size();
    }
};
std::mutex g_digest_mu;
std::list<DigestEntry> g_digest_cache;  // front: most recently used
constexpr size_t DIGEST_CACHE_BYTES = 512ull << 20;

// the desc's matrix data as a cache entry (copies)
DigestEntry digest_key(const neo_ccs_desc* d) {
    DigestEntry e;
    e.n = d->n; e.m = d->m; e.t = d->t;
    e.ident.assign(d->is_identity, d->is_identity + d->t);
    e.nnz_off.assign(d->nnz_off, d->nnz_off + d->t + 1);
    const uint64_t nnz = d->nnz_off[d->t];
    for (uint32_t j = 0; j < d->t; j++) {
        if (d->is_identity[j]) continue;
        const uint64_t* cp = d->col_ptr + (size_t)j * (d->m + 1);
        e.col_ptr.insert(e.col_ptr.end(), cp, cp + d->m + 1);
    }
    e.row_idx.assign(d->row_idx, d->row_idx + nnz);
    e.vals.assign(d->vals, d->vals + nnz);
    return e;
}

bool digest_key_eq(const DigestEntry& a, const DigestEntry& b) {
    return a.n == b.n && a.m == b.m && a.t == b.t && a.ident == b.ident && a.nnz_off == b.nnz_off &&
           a.col_ptr == b.col_ptr && a.row_idx == b.row_idx && a.vals == b.vals;
}
}  // namespace

static void ccs_digest_compute(const neo_ccs_desc* d, uint64_t* out4);

static void ccs_digest_words(const neo_ccs_desc* d, uint64_t* out4) {
    DigestEntry key = digest_key(d);
    {
        std::lock_guard<std::mutex> lk(g_digest_mu);
        for (auto it = g_digest_cache.begin(); it != g_digest_cache.end(); ++it)
            if (digest_key_eq(*it, key)) {
                memcpy(out4, it->out, 32);
                g_digest_cache.splice(g_digest_cache.begin(), g_digest_cache, it);
                return;
            }
    }
    ccs_digest_compute(d, out4);
    if (key.bytes() > DIGEST_CACHE_BYTES) return;
    memcpy(key.out, out4, 32);
    std::lock_guard<std::mutex> lk(g_digest_mu);
    g_digest_cache.push_front(std::move(key));
    size_t total = 0;
    for (auto& e : g_digest_cache) total += e.bytes();
    while (total > DIGEST_CACHE_BYTES && g_digest_cache.size() > 1) {
        total -= g_digest_cache.back().bytes();
        g_digest_cache.pop_back();
    }
}

// Row-major (column, value) list of matrix j: columns ascending within a row
// (the order of the dense scan the reference's digest follows).
static std::vector<std::pair<uint64_t, uint64_t>> ccs_row_major(const neo_ccs_desc* d, uint32_t j,
                                                                std::vector<uint64_t>& off) {
    const uint64_t* cp = d->col_ptr + (size_t)j * (d->m + 1);
    const uint64_t base = d->nnz_off[j], nnz = d->nnz_off[j + 1] - base;
    off.assign(d->n + 1, 0);
    for (uint64_t k = 0; k < nnz; k++) off[d->row_idx[base + k] + 1]++;
    for (uint32_t r = 0; r < d->n; r++) off[r + 1] += off[r];
    std::vector<std::pair<uint64_t, uint64_t>> ent(nnz);
    std::vector<uint64_t> wp(off.begin(), off.end() - 1);
    for (uint32_t c = 0; c < d->m; c++)
        for (uint64_t k = cp[c]; k < cp[c + 1]; k++) ent[wp[d->row_idx[base + k]]++] = {c, d->vals[base + k]};
    return ent;
}

static void ccs_digest_compute(const neo_ccs_desc* d, uint64_t* out4) {
    const neo::Poseidon2W16& P = neo::digest_perm();
    // the sponge is one sequential chain; the row-major reorder of each sparse
    // matrix runs on a helper thread meanwhile (matrix j is ready while the
    // sponge absorbs matrices 0..j-1)
    struct RowMajor {
        std::vector<uint64_t> off;
        std::vector<std::pair<uint64_t, uint64_t>> ent;
    };
    std::vector<RowMajor> rm(d->t);
    std::vector<std::future<void>> ready(d->t);
    for (uint32_t j = 0; j < d->t; j++)
        if (!d->is_identity[j])
        {
            auto task = [d, j, &rm] { rm[j].ent = ccs_row_major(d, j, rm[j].off); };
            try {
                ready[j] = std::async(std::launch::async, task);
            } catch (const std::system_error&) {  // no thread to spare: reorder when the sponge needs it
                ready[j] = std::async(std::launch::deferred, task);
            }
        }
    uint64_t st[16] = {0};
    int ab = 0;
    const char* dom = "neo/ccs/matrices/v1";
    for (const char* c = dom; *c; c++) {
        if (ab >= 15) { P.permute(st); ab = 0; }
        st[ab++] = (uint8_t)*c;
    }
    if (ab + 3 >= 16) { P.permute(st); ab = 0; }
    st[ab] = d->n; st[ab + 1] = d->m; st[ab + 2] = d->t;
    P.permute(st);
    for (uint32_t j = 0; j < d->t; j++) {
        ab = 0;
        st[ab++] = j;
        auto emit = [&](uint64_t row, uint64_t col, uint64_t val) {
            if (ab + 3 > 15) { P.permute(st); ab = 0; }
            st[ab] = row; st[ab + 1] = col; st[ab + 2] = gl::canon(val);
            ab += 3;
        };
        if (d->is_identity[j]) {
            for (uint64_t r = 0; r < d->n; r++) emit(r, r, 1);
        } else {
            ready[j].get();
            const auto& off = rm[j].off;
            const auto& ent = rm[j].ent;
            for (uint32_t r = 0; r < d->n; r++)
                for (uint64_t e = off[r]; e < off[r + 1]; e++) emit(r, ent[e].first, ent[e].second);
            rm[j] = RowMajor();
        }
        P.permute(st);
    }
    for (int i = 0; i < 4; i++) out4[i] = st[i];
}

// digest_fields (crates/neo-fold/src/memory_sidecar/transcript.rs:4-10)
static void digest_fields(const char* label, const std::vector<uint64_t>& fs, uint8_t out[32]) {
    neo::Transcript h("memory/public_digest");
    h.append_message("digest/label", label);
    auto n = le64(fs.size());
    h.append_message("digest/len", n.data(), 8);
    std::vector<uint64_t> c(fs.size());
    for (size_t i = 0; i < fs.size(); i++) c[i] = gl::canon(fs[i]);
    h.append_fields("digest/fields", c.data(), c.size());
    h.digest32(out);
}

// MemInit of a Twist instance (crates/neo-memory/src/mem_init.rs): Sparse pairs
// in canonical form (strictly increasing addresses < 2^ell_addr) or Zero, and
// the public digest absorbed per step (digest_fields "twist/init/sparse" /
// "twist/init/zero", memory_sidecar/memory.rs:86-124).  false: not canonical.
static bool twist_set_init(TwistInst& ti, uint64_t n, const uint64_t* addr, const uint64_t* val) {
    std::vector<uint64_t> a, v, fs;
    for (uint64_t e = 0; e < n; e++) {
        if (addr[e] >> ti.ea) return false;
        if (e && addr[e] <= addr[e - 1]) return false;
        a.push_back(addr[e]);
        v.push_back(gl::canon(val[e]));
        fs.push_back(addr[e]);
        fs.push_back(gl::canon(val[e]));
    }
    ti.init_addr.swap(a);
    ti.init_val.swap(v);
    digest_fields(n ? "twist/init/sparse" : "twist/init/zero", fs, ti.digest);
    return true;
}


static int neo_ccs_digest_impl_abi(const neo_ccs_desc* d, uint64_t* out4) {
    if (!d || !out4 || d->t == 0 || d->n == 0 || d->m == 0) return NEO_ERR_ARG;
    ccs_digest_words(d, out4);
    return NEO_OK;
}
extern "C" int neo_ccs_digest(const neo_ccs_desc* d, uint64_t* out4) { NEO_ABI_GUARD(neo_ccs_digest_impl_abi(d, out4)) }

static int shard_create_impl(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, uint32_t m_in, uint32_t k_rho,
                             const char* app_label, const neo_mem_desc* mem, neo_gpu_shard** out) {
    if (!ctx) return NEO_ERR_ARG;
    if (!desc || !out || !app_label) return ctx->fail(NEO_ERR_ARG, "shard_create: null argument");
    *out = nullptr;
    if (desc->n != desc->m || desc->n < 2 || (desc->n & (desc->n - 1)))
        return ctx->fail(NEO_ERR_UNSUPPORTED, "shard_create: requires n == m == power of two");
    PPEntry* pp = pp_lookup(ctx->device, desc->m);
    if (!pp) return ctx->fail(NEO_ERR_ARG, "shard_create: upload PP for this m first");
    if (k_rho == 0 || k_rho > 17 || m_in == 0 || m_in > desc->m) return ctx->fail(NEO_ERR_ARG, "shard_create: k_rho/m_in");
    cudaSetDevice(ctx->device);
    auto* sh = new neo_gpu_shard();
    std::unique_ptr<neo_gpu_shard> guard(sh);
    sh->ctx = ctx;
    int rc = dev_ccs_upload(ctx, desc, sh->ccs);
    if (rc) return rc;
    sh->n = desc->n; sh->m = desc->m; sh->m32 = desc->m; sh->t = desc->t; sh->m_in = m_in; sh->k_rho = k_rho;
    sh->kappa = pp->kappa;
    if (sh->t > 4) return ctx->fail(NEO_ERR_UNSUPPORTED, "shard_create: t <= 4 supported by the fold step");
    while ((1u << sh->ell_n) < sh->n) sh->ell_n++;
    int fdeg = 0;
    for (uint32_t tt = 0; tt < desc->n_terms; tt++) {
        int dg = 0;
        for (uint32_t j = 0; j < desc->t; j++) dg += desc->f_exps[tt * desc->t + j];
        fdeg = std::max(fdeg, dg);
    }
    sh->d_sc = std::max<uint32_t>(fdeg + 1, 2 * sh->b + 2);
    header_params(sh);
    ccs_digest_words(desc, sh->mat_digest);
    sh->tr.reset(new neo::Transcript(app_label));
    const uint64_t m = sh->m;
    const uint64_t L = 1ULL << sh->ell_n;
    // ---- memory instances and the bus layout (neo-memory/src/cpu/bus_layout.rs:91-190) ----
    if (mem && (mem->n_shout || mem->n_twist)) {
        if ((mem->n_shout && !mem->shout) || (mem->n_twist && !mem->twist))
            return ctx->fail(NEO_ERR_ARG, "shard_create: null memory instance array");
        if (mem->steps == 0) return ctx->fail(NEO_ERR_ARG, "shard_create: memory steps must be >= 1");
        uint32_t col = 0;
        for (uint32_t i = 0; i < mem->n_shout; i++) {
            const neo_mem_instance& s = mem->shout[i];
            if (s.ell_addr == 0 || s.ell_addr > 24) return ctx->fail(NEO_ERR_UNSUPPORTED, "shard_create: Shout ell_addr in 1..24");
            if (i && s.ell_addr != mem->shout[0].ell_addr)
                return ctx->fail(NEO_ERR_ARG, "shard_create: Shout instances need one ell_addr (batched addr-pre)");
            if (s.table_len && !s.table) return ctx->fail(NEO_ERR_ARG, "shard_create: Shout table is null");
            auto si = std::make_unique<ShoutInst>();
            si->ea = s.ell_addr; si->k = s.k; si->d = s.d; si->n_side = s.n_side; si->ell = s.ell;
            si->table.assign(s.table, s.table + s.table_len);
            digest_fields("shout/table", si->table, si->digest);
            const uint64_t P = 1ULL << s.ell_addr;
            std::vector<K> tk(P, gl::kzero());
            for (uint64_t a = 0; a < P && a < s.table_len; a++) tk[a] = gl::kfq(gl::canon(s.table[a]));
            NEO_CK(ctx, si->d_table.alloc(P));
            NEO_CK(ctx, cudaMemcpyAsync(si->d_table.p, tk.data(), P * sizeof(K), cudaMemcpyHostToDevice, ctx->stream));
            si->col0 = col;
            col += s.ell_addr + 2;
            sh->shout.push_back(std::move(si));
        }
        for (uint32_t i = 0; i < mem->n_twist; i++) {
            const neo_mem_instance& w = mem->twist[i];
            if (w.ell_addr == 0 || w.ell_addr > 24) return ctx->fail(NEO_ERR_UNSUPPORTED, "shard_create: Twist ell_addr in 1..24");
            if (w.n_init && (!w.init_addr || !w.init_val)) return ctx->fail(NEO_ERR_ARG, "shard_create: Twist init is null");
            auto ti = std::make_unique<TwistInst>();
            ti->ea = w.ell_addr; ti->k = w.k; ti->d = w.d; ti->n_side = w.n_side; ti->ell = w.ell;
            if (!twist_set_init(*ti, w.n_init, w.init_addr, w.init_val))
                return ctx->fail(NEO_ERR_ARG, "shard_create: Twist init must have strictly increasing addresses < 2^ell_addr");
            ti->col0 = col;
            col += 2 * w.ell_addr + 5;
            sh->twist.push_back(std::move(ti));
        }
        sh->steps = mem->steps;
        sh->bus_cols = col;
        const uint64_t region = (uint64_t)col * mem->steps;
        if (region > m || m - region < m_in) return ctx->fail(NEO_ERR_ARG, "shard_create: bus region overlaps the public inputs");
        if (m_in + mem->steps > sh->n) return ctx->fail(NEO_ERR_ARG, "shard_create: bus time rows out of range");
        sh->bus_base = m - region;
        uint32_t max_asm = 2;
        for (auto& s : sh->shout) max_asm = std::max(max_asm, s->ea + 1);
        for (auto& w : sh->twist) max_asm = std::max(max_asm, 2 * w->ea + 4);
        NEO_CK(ctx, sh->d_cols.alloc((size_t)col * L));
        NEO_CK(ctx, sh->d_prev_cols.alloc((size_t)col * L));
        size_t asm_len = (size_t)max_asm * L;
        for (auto& s : sh->shout) asm_len = std::max<size_t>(asm_len, 2ULL << s->ea);
        NEO_CK(ctx, sh->d_asm.alloc(asm_len));
        NEO_CK(ctx, sh->d_busw.alloc(mem->steps));
        NEO_CK(ctx, sh->d_busy.alloc((size_t)std::max<uint32_t>(1 + k_rho, 2) * col * NEO_D));
        NEO_CK(ctx, sh->d_r.alloc(std::max<uint32_t>(sh->ell_n, 32)));
        NEO_CK(ctx, sh->d_chi.alloc(L));
        NEO_CK(ctx, sh->d_vj.alloc((size_t)sh->t * m));
        NEO_CK(ctx, sh->d_yv.alloc((size_t)std::max<uint32_t>(k_rho, 2) * sh->t * NEO_D));
        NEO_CK(ctx, sh->d_yvsc.alloc((size_t)std::max<uint32_t>(k_rho, 2) * sh->t));
        NEO_CK(ctx, sh->valwit.alloc((size_t)2 * NEO_D * m));
        NEO_CK(ctx, sh->valplanes.alloc((size_t)k_rho * NEO_D * m));
        for (auto& s : sh->shout) (void)s;
        size_t wmax = 1;
        for (auto& s : sh->shout) wmax = std::max<size_t>(wmax, 1ULL << s->ea);
        NEO_CK(ctx, sh->d_w.alloc(wmax));
    }
    NEO_CK(ctx, sh->Zall.alloc((size_t)(1 + k_rho) * NEO_D * m));
    NEO_CK(ctx, sh->d_z.alloc(m));
    NEO_CK(ctx, sh->d_mix.alloc((size_t)NEO_D * m));
    NEO_CK(ctx, sh->d_rot.alloc((size_t)(1 + k_rho) * NEO_D * RLC_ROT_ROW));
    NEO_CK(ctx, sh->d_commits.alloc((size_t)(1 + k_rho) * sh->kappa * NEO_D));
    NEO_CK(ctx, sh->d_flags.alloc(2));
    NEO_CK(ctx, sh->d_ychild.alloc((size_t)k_rho * sh->t * NEO_D));
    size_t mixv = (size_t)(1 + k_rho) * std::max<uint32_t>(sh->kappa, 2 * sh->t + m_in) * NEO_D * 2;
    NEO_CK(ctx, sh->d_mixv.alloc(mixv));
    NEO_CK(ctx, sh->d_mixo.alloc(mixv));
    *out = guard.release();
    return NEO_OK;
}

static int neo_gpu_shard_create_impl_abi(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, uint32_t m_in, uint32_t k_rho,
                                    const char* app_label, neo_gpu_shard** out) {
    return shard_create_impl(ctx, desc, m_in, k_rho, app_label, nullptr, out);
}
extern "C" int neo_gpu_shard_create(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, uint32_t m_in, uint32_t k_rho,
                                    const char* app_label, neo_gpu_shard** out) { NEO_ABI_GUARD(neo_gpu_shard_create_impl_abi(ctx, desc, m_in, k_rho, app_label, out)) }

static int neo_gpu_shard_create_mem_impl_abi(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, uint32_t m_in, uint32_t k_rho,
                                        const char* app_label, const neo_mem_desc* mem, neo_gpu_shard** out) {
    return shard_create_impl(ctx, desc, m_in, k_rho, app_label, mem, out);
}
extern "C" int neo_gpu_shard_create_mem(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, uint32_t m_in, uint32_t k_rho,
                                        const char* app_label, const neo_mem_desc* mem, neo_gpu_shard** out) { NEO_ABI_GUARD(neo_gpu_shard_create_mem_impl_abi(ctx, desc, m_in, k_rho, app_label, mem, out)) }

static int neo_gpu_shard_destroy_impl_abi(neo_gpu_shard* sh) {
    if (!sh) return NEO_ERR_ARG;
    cudaSetDevice(sh->ctx->device);
    cudaStreamSynchronize(sh->ctx->stream);
    if (sh->orc) neo_gpu_ccs_oracle_destroy(sh->orc);
    for (auto* o : sh->mem_slots) neo_gpu_mem_oracle_destroy(o);
    for (auto* o : sh->ta_slots) neo_gpu_twist_addr_destroy(o);
    delete sh;
    return NEO_OK;
}
extern "C" int neo_gpu_shard_destroy(neo_gpu_shard* sh) { NEO_ABI_GUARD(neo_gpu_shard_destroy_impl_abi(sh)) }

// ---------------------------------------------------------------------------
// one fold step
// ---------------------------------------------------------------------------
int ccs_oracle_create_dev(neo_gpu_ctx* ctx, const DevCcs* ccs, const int8_t* d_Z, uint32_t k, uint32_t b,
                          const K* alpha, const K* beta_a, const K* beta_r, K gamma, const K* r_inputs,
                          uint32_t ell_d, uint32_t ell_n, uint32_t d_sc, neo_gpu_ccs_oracle** out);
int ccs_oracle_dev_vj(neo_gpu_ccs_oracle* o, const K** vj);
int ccs_oracle_round_launch(neo_gpu_ccs_oracle* o, K* d_dst, uint32_t* ncoef);
void ccs_oracle_round_set(neo_gpu_ccs_oracle* o, const K* coeffs);
bool mem_round_multi_ok(const neo_gpu_mem_oracle* o);
int ta_round_launch(neo_gpu_twist_addr* o, K* d_dst, bool* launched);
int mem_claims_multi(neo_gpu_ctx* ctx, neo_gpu_mem_oracle* const* os, int n, K* claims, DevBuf<K>& partials,
                     DevBuf<K>& d_slots, HostBuf<K>& h_slots);
int mem_round_launch_multi(neo_gpu_ctx* ctx, neo_gpu_mem_oracle* const* os, int n, K* const* d_out,
                           DevBuf<K>& partials);

namespace {

static void interpolate(const std::vector<K>& xs, const std::vector<K>& ys, std::vector<K>& co) {
    // sumcheck.rs:74-118; the nodes here are always 0..n-1, whose Lagrange
    // denominators 1 / prod_{j != i} (i - j) are computed once per n
    const size_t n = xs.size();
    bool ints = true;
    for (size_t i = 0; i < n; i++) ints &= xs[i].im == 0 && xs[i].re == i;
    static thread_local std::vector<std::vector<K>> inv_den;
    if (ints && inv_den.size() <= n) inv_den.resize(n + 1);
    if (ints && inv_den[n].empty()) {
        inv_den[n].resize(n);
        for (size_t i = 0; i < n; i++) {
            K den = gl::kone();
            for (size_t j = 0; j < n; j++)
                if (i != j) den = gl::kmul(den, gl::ksub(xs[i], xs[j]));
            inv_den[n][i] = gl::kinv(den);
        }
    }
    co.assign(n, gl::kzero());
    std::vector<K> numer(n), next(n);
    for (size_t i = 0; i < n; i++) {
        std::fill(numer.begin(), numer.end(), gl::kzero());
        numer[0] = gl::kone();
        size_t cur = 0;
        for (size_t j = 0; j < n; j++) {
            if (i == j) continue;
            std::fill(next.begin(), next.end(), gl::kzero());
            for (size_t d = 0; d <= cur; d++) {
                next[d + 1] = gl::kadd(next[d + 1], numer[d]);
                next[d] = gl::kadd(next[d], gl::kmul(gl::kneg(xs[j]), numer[d]));
            }
            numer.swap(next);
            cur++;
        }
        K sc;
        if (ints) {
            sc = gl::kmul(ys[i], inv_den[n][i]);
        } else {
            K den = gl::kone();
            for (size_t j = 0; j < n; j++)
                if (i != j) den = gl::kmul(den, gl::ksub(xs[i], xs[j]));
            sc = gl::kmul(ys[i], gl::kinv(den));
        }
        for (size_t d = 0; d <= cur; d++) co[d] = gl::kadd(co[d], gl::kmul(sc, numer[d]));
    }
}

static K poly_eval(const std::vector<K>& c, K x) {
    K r = c.back();
    for (int d = (int)c.size() - 2; d >= 0; d--) r = gl::kadd(gl::kmul(r, x), c[d]);
    return r;
}

static void absorb_k(neo::Transcript& tr, const char* label, K v) {
    uint64_t f[2] = {v.re, v.im};
    tr.append_fields(label, f, 2);
}

static std::vector<uint64_t> k_flat(const std::vector<K>& v) {
    std::vector<uint64_t> f(2 * v.size());
    for (size_t i = 0; i < v.size(); i++) { f[2 * i] = v[i].re; f[2 * i + 1] = v[i].im; }
    return f;
}

static inline bool keq(K a, K b) { return a.re == b.re && a.im == b.im; }
static inline void push_k(std::vector<uint64_t>& P, K v) { P.push_back(v.re); P.push_back(v.im); }

// One claim of a batched sum-check: a GPU round oracle of one of three families.
struct Claim {
    std::string label;
    uint32_t deg = 0;
    bool dyn = true;
    K sum{};
    neo_gpu_ccs_oracle* ccs = nullptr;
    neo_gpu_mem_oracle* mem = nullptr;
    neo_gpu_twist_addr* ta = nullptr;
    int evals(const K* xs, uint32_t nx, K* ys) const {
        if (ccs) return neo_gpu_ccs_oracle_evals(ccs, (const uint64_t*)xs, nx, (uint64_t*)ys);
        if (mem) return neo_gpu_mem_oracle_evals(mem, (const uint64_t*)xs, nx, (uint64_t*)ys);
        return neo_gpu_twist_addr_evals(ta, (const uint64_t*)xs, nx, (uint64_t*)ys);
    }
    int fold(K r) const {
        if (ccs) return neo_gpu_ccs_oracle_fold(ccs, (const uint64_t*)&r);
        if (mem) return neo_gpu_mem_oracle_fold(mem, (const uint64_t*)&r);
        return neo_gpu_twist_addr_fold(ta, (const uint64_t*)&r);
    }
};

// run_batched_sumcheck_prover (sumcheck.rs:350-456) inside sc_start / sc_end
// (sumcheck_ds.rs:11-19); round polynomials appended to P in claim order.
// Per round every claim is launched first -- the Pi_CCS claim writes its
// coefficients, the memory claims their values at 0..deg (all of them in one
// multi-claim fold and eval), the Twist address-lane claims theirs at 0, 1,
// 2, into one device array -- then a single copy and sync bring the round
// back; claims whose tables are exhausted take the per-claim path.
static int run_batched_ds(neo_gpu_shard* sh, const char* domain, uint64_t inst_idx, std::vector<Claim>& cl,
                          uint32_t rounds, std::vector<K>& chals, std::vector<K>& finals, std::vector<uint64_t>& P,
                          BatchRec* rec = nullptr) {
    neo_gpu_ctx* ctx = sh->ctx;
    neo::Transcript& tr = *sh->tr;
    auto bi = le64(inst_idx);
    tr.append_message("sc/domain", domain);
    tr.append_message("sc/inst_idx", bi.data(), 8);
    std::vector<K> running(cl.size());
    for (size_t i = 0; i < cl.size(); i++) running[i] = cl[i].sum;
    std::vector<std::vector<K>> polys(cl.size());
    if (rec) {
        *rec = BatchRec();
        for (auto& c : cl) {
            rec->labels.push_back(c.label);
            rec->degs.push_back(c.deg);
            rec->sums.push_back(c.sum);
        }
        rec->polys.assign(cl.size(), {});
    }
    // slots: MAX_SLOT K values per claim
    constexpr uint32_t MAX_SLOT = 33;
    NEO_CK(ctx, sh->d_round.ensure(cl.size() * MAX_SLOT));
    NEO_CK(ctx, sh->h_round.ensure(cl.size() * MAX_SLOT));
    chals.clear();
    std::vector<neo_gpu_mem_oracle*> mos;
    std::vector<K*> mdst;
    std::vector<uint32_t> kind(cl.size()), ncoef(cl.size());  // kind: 0 per-claim, 1 ccs, 2 multi memory
    for (uint32_t rd = 0; rd < rounds; rd++) {
        auto br = le64(rd);
        tr.append_message("batched/round_idx", br.data(), 8);
        mos.clear();
        mdst.clear();
        for (size_t i = 0; i < cl.size(); i++) {
            K* slot = sh->d_round.p + i * MAX_SLOT;
            kind[i] = 0;
            if (cl[i].ccs && cl[i].deg + 1 <= MAX_SLOT) {
                int rc = ccs_oracle_round_launch(cl[i].ccs, slot, &ncoef[i]);
                if (rc) return rc;
                kind[i] = 1;
            } else if (cl[i].mem && cl[i].deg + 1 <= MAX_SLOT && neo_gpu_mem_oracle_degree_bound(cl[i].mem) == cl[i].deg &&
                       mem_round_multi_ok(cl[i].mem)) {
                mos.push_back(cl[i].mem);
                mdst.push_back(slot);
                kind[i] = 2;
            } else if (cl[i].ta && cl[i].deg == 2) {
                bool launched = false;
                int rc = ta_round_launch(cl[i].ta, slot, &launched);
                if (rc) return rc;
                if (launched) kind[i] = 2;  // values at 0, 1, 2 in the slot
            }
        }
        for (size_t i0 = 0; i0 < mos.size(); i0 += 24) {
            const int nn = (int)std::min<size_t>(24, mos.size() - i0);
            int rc = mem_round_launch_multi(ctx, mos.data() + i0, nn, mdst.data() + i0, sh->d_mpart);
            if (rc) return rc;
        }
        NEO_CK(ctx, cudaMemcpyAsync(sh->h_round.p, sh->d_round.p, cl.size() * MAX_SLOT * sizeof(K),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        NEO_CK(ctx, ctx_sync(ctx));
        for (size_t i = 0; i < cl.size(); i++) {
            const uint32_t np = cl[i].deg + 1;
            std::vector<K> xs(np), ys(np);
            for (uint32_t x = 0; x < np; x++) xs[x] = gl::kfq(x);
            const K* h = sh->h_round.p + i * MAX_SLOT;
            if (kind[i] == 1) {
                // values at 0..deg from the coefficients (Horner, sumcheck.rs:48-60)
                ccs_oracle_round_set(cl[i].ccs, h);
                std::vector<K> co(h, h + ncoef[i]);
                for (uint32_t x = 0; x < np; x++) ys[x] = poly_eval(co, xs[x]);
            } else if (kind[i] == 2) {
                for (uint32_t x = 0; x < np; x++) ys[x] = h[x];
            } else {
                int rc = cl[i].evals(xs.data(), np, ys.data());
                if (rc) return rc;
            }
            if (!keq(gl::kadd(ys[0], ys[1]), running[i]))
                return ctx->fail(NEO_ERR_INVARIANT, ("batched sum-check " + cl[i].label + ": p(0)+p(1) != running sum").c_str());
            interpolate(xs, ys, polys[i]);
        }
        for (size_t i = 0; i < cl.size(); i++) {
            tr.append_message("batched/claim_label", cl[i].label);
            auto bc = le64(i);
            tr.append_message("batched/claim_idx", bc.data(), 8);
            for (auto& c : polys[i]) absorb_k(tr, "batched/round/coeff", c);
        }
        uint64_t c0 = tr.challenge_field("batched/challenge/0");
        uint64_t c1 = tr.challenge_field("batched/challenge/1");
        K r = gl::kmk(c0, c1);
        chals.push_back(r);
        for (size_t i = 0; i < cl.size(); i++) {
            running[i] = poly_eval(polys[i], r);
            int rc = cl[i].fold(r);
            if (rc) return rc;
            for (auto& c : polys[i]) push_k(P, c);
            if (rec) rec->polys[i].push_back(polys[i]);
        }
    }
    tr.append_message("sc/domain_end", domain);
    tr.append_message("sc/inst_idx_end", bi.data(), 8);
    finals = running;
    if (rec) {
        rec->chals = chals;
        rec->finals = finals;
    }
    return NEO_OK;
}

// bind_batched_claim_sums (memory_sidecar/transcript.rs:12-26)
static void bind_claim_sums(neo::Transcript& tr, const char* prefix, const std::vector<K>& sums,
                            const std::vector<std::string>& labels) {
    auto n = le64(sums.size());
    tr.append_message(prefix, n.data(), 8);
    for (size_t i = 0; i < sums.size(); i++) {
        tr.append_message("addr_batch/label", labels[i]);
        auto bi = le64(i);
        tr.append_message("addr_batch/idx", bi.data(), 8);
        absorb_k(tr, "addr_batch/claimed_sum", sums[i]);
    }
}

// sample_ext_point (neo-memory/src/ts_common.rs:22-37)
static std::vector<K> sample_ext_point(neo::Transcript& tr, const char* label, const char* l0, const char* l1,
                                       uint32_t n) {
    std::vector<K> out;
    for (uint32_t i = 0; i < n; i++) {
        auto b8 = le64(i);
        tr.append_message(label, b8.data(), 8);
        uint64_t c0 = tr.challenge_field(l0);
        uint64_t c1 = tr.challenge_field(l1);
        out.push_back(gl::kmk(c0, c1));
    }
    return out;
}

// bitness_weights (memory_sidecar/utils.rs:43-71)
static std::vector<K> bitness_weights(K r0, uint32_t n, uint64_t sep) {
    K base = gl::kadd(r0, gl::kfq(gl::canon(sep)));
    if (keq(base, gl::kzero()) || keq(base, gl::kone()) || keq(base, gl::kneg(gl::kone())))
        base = gl::kadd(base, gl::kone());
    if (keq(base, gl::kzero())) base = gl::kone();
    std::vector<K> w;
    K cur = gl::kone();
    for (uint32_t i = 0; i < n; i++) {
        w.push_back(cur);
        cur = gl::kmul(cur, base);
    }
    return w;
}

// bus openings of n_w consecutive digit witnesses (stride 54*m) at the point
// already in sh->d_r: y rows appended to the host vectors (bus_cols x 54 K per
// witness) and their base-b scalars.
static int bus_openings(neo_gpu_shard* sh, const int8_t* d_Z, uint32_t n_w, std::vector<K>& y, std::vector<K>& ysc) {
    neo_gpu_ctx* ctx = sh->ctx;
    const uint32_t nb = sh->bus_cols;
    bus_weights_kernel<<<ceil_div(sh->steps, 256), 256, 0, ctx->stream>>>(sh->d_r.p, sh->ell_n, sh->m_in, sh->steps,
                                                                          sh->d_busw.p);
    NEO_LAUNCHED(ctx);
    const uint64_t items = (uint64_t)n_w * nb * NEO_D;
    bus_open_kernel<<<(unsigned)ceil_div(items, BUS_OPEN_WARPS), 32 * BUS_OPEN_WARPS, 0, ctx->stream>>>(
        d_Z, sh->m, sh->bus_base, sh->steps, nb, items, sh->d_busw.p, sh->d_busy.p);
    NEO_LAUNCHED(ctx);
    y.resize((size_t)n_w * nb * NEO_D);
    NEO_CK(ctx, ctx_d2h(ctx, y.data(), sh->d_busy.p, y.size() * sizeof(K)));
    NEO_CK(ctx, ctx_sync(ctx));
    ysc.assign((size_t)n_w * nb, gl::kzero());
    for (size_t q = 0; q < (size_t)n_w * nb; q++) {
        K s = gl::kzero();
        uint64_t pw = 1;
        for (int rho = 0; rho < NEO_D; rho++) {
            s = gl::kadd(s, gl::kscale(y[q * NEO_D + rho], pw));
            pw = gl::mul(pw, sh->b);
        }
        ysc[q] = s;
    }
    return NEO_OK;
}

static int upload_point(neo_gpu_shard* sh, const std::vector<K>& r) {
    NEO_CK(sh->ctx, cudaMemcpyAsync(sh->d_r.p, r.data(), r.size() * sizeof(K), cudaMemcpyHostToDevice, sh->ctx->stream));
    return NEO_OK;
}

// gather bus columns (ids) of `src` into d_asm, in the given order
static int assemble(neo_gpu_shard* sh, const K* src, const std::vector<uint32_t>& ids) {
    const uint64_t L = 1ULL << sh->ell_n;
    for (size_t i = 0; i < ids.size(); i++)
        NEO_CK(sh->ctx, cudaMemcpyAsync(sh->d_asm.p + i * L, src + (size_t)ids[i] * L, L * sizeof(K),
                                        cudaMemcpyDeviceToDevice, sh->ctx->stream));
    return NEO_OK;
}

static std::vector<uint32_t> twist_read_ids(const TwistInst& w) {
    std::vector<uint32_t> v = {w.col0 + 2 * w.ea, w.col0 + 2 * w.ea + 3};  // has_read, rv
    for (uint32_t b = 0; b < w.ea; b++) v.push_back(w.col0 + b);            // ra bits
    v.push_back(w.col0 + 2 * w.ea + 1);                                     // has_write
    v.push_back(w.col0 + 2 * w.ea + 4);                                     // inc
    for (uint32_t b = 0; b < w.ea; b++) v.push_back(w.col0 + w.ea + b);     // wa bits
    return v;
}
static std::vector<uint32_t> twist_write_ids(const TwistInst& w) {
    std::vector<uint32_t> v = {w.col0 + 2 * w.ea + 1, w.col0 + 2 * w.ea + 2, w.col0 + 2 * w.ea + 4};  // hw, wv, inc
    for (uint32_t b = 0; b < w.ea; b++) v.push_back(w.col0 + w.ea + b);
    return v;
}
static std::vector<uint32_t> twist_val_ids(const TwistInst& w) {
    std::vector<uint32_t> v = {w.col0 + 2 * w.ea + 1, w.col0 + 2 * w.ea + 4};  // hw, inc
    for (uint32_t b = 0; b < w.ea; b++) v.push_back(w.col0 + w.ea + b);
    return v;
}

// prove_rlc_dec_lane (shard.rs:1170-1331): bind inputs, sample rhos, mix,
// split into k_rho planes (d_planes), commit, child ME claims at r (core rows
// from vj, bus rows from the planes), DEC public checks.
static int rlc_dec_lane(neo_gpu_shard* sh, const char* lane, uint32_t idx, const std::vector<MeInst>& ins,
                        const int8_t* d_wits, int8_t* d_planes, const std::vector<K>& r, const K* d_vj,
                        const uint8_t* digest, std::vector<MeInst>& children, std::vector<uint64_t>& P,
                        LaneRec* rec = nullptr) {
    neo_gpu_ctx* ctx = sh->ctx;
    neo::Transcript& tr = *sh->tr;
    const uint32_t k = (uint32_t)ins.size(), t = sh->t, kappa = sh->kappa, nb = sh->bus_cols;
    const uint32_t d_pad = 1u << sh->ell_d;
    const uint64_t m = sh->m;
    int rc;
    tr.append_message("fold/rlc_inputs/v1", lane);
    uint64_t si = idx, mc = k;
    tr.append_u64s("step_idx", &si, 1);
    tr.append_u64s("me_count", &mc, 1);
    for (auto& me : ins) {
        tr.append_fields("c_data", me.c.data(), me.c.size());
        uint64_t mi = me.m_in;
        tr.append_u64s("m_in", &mi, 1);
        tr.append_message("me_fold_digest", me.digest, 32);
        for (auto& rl : me.r) absorb_k(tr, "r_limb", rl);
        tr.append_fields("X", me.X.data(), me.X.size());
        for (auto& ye : me.y) absorb_k(tr, "y_elem", ye);
        for (auto& ys_ : me.ysc) absorb_k(tr, "y_scalar", ys_);
        uint64_t zero = 0;
        tr.append_u64s("c_step_coords_len", &zero, 1);
        tr.append_fields("c_step_coords", nullptr, 0);
        tr.append_u64s("u_offset", &zero, 1);
        tr.append_u64s("u_len", &zero, 1);
    }
    // sample_rot_rhos_n (common.rs:467-573) with draw_alphabet_vector (common.rs:432-465)
    std::vector<int8_t> rhos((size_t)k * NEO_D);
    static const int8_t A5[5] = {-2, -1, 0, 1, 2};
    for (uint32_t i = 0; i < k; i++) {
        auto bi = le64(i);
        tr.append_message("rlc/rot/index", bi.data(), 8);
        const uint32_t bucket = (1u << 16) / 5 * 5;
        uint64_t ctr = i;
        size_t got = 0;
        while (got < NEO_D) {
            auto bc = le64(ctr);
            tr.append_message("rlc/rot/chunk", bc.data(), 8);
            uint8_t dig[32];
            tr.digest32(dig);
            for (int w = 0; w < 16 && got < NEO_D; w++) {
                uint32_t xv = (uint32_t)dig[2 * w] | ((uint32_t)dig[2 * w + 1] << 8);
                if (xv < bucket) rhos[(size_t)i * NEO_D + got++] = A5[xv % 5];
            }
            ctr++;
        }
    }
    for (auto v : rhos) P.push_back(gl::from_i64(v));
    // Z_mix = sum rho_i Z_i (count == 1: identity)
    if ((rc = rlc_mix_device(ctx, rhos.data(), d_wits, k, m, sh->d_mix.p, sh->d_rot.p))) return rc;
    // parent commitment and core y: rot mixes of the k commitments / y vectors
    std::vector<uint64_t> c_parent((size_t)kappa * NEO_D);
    std::vector<K> y_parent((size_t)t * NEO_D);
    {
        std::vector<uint64_t> cv((size_t)k * kappa * NEO_D);
        for (uint32_t i = 0; i < k; i++) memcpy(&cv[(size_t)i * kappa * NEO_D], ins[i].c.data(), kappa * NEO_D * 8);
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_mixv.p, cv.data(), cv.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
        rot_mix_kernel<<<kappa, dim3(64, 16), 0, ctx->stream>>>(sh->d_rot.p, k, sh->d_mixv.p, kappa, 1, sh->d_mixo.p);
        NEO_LAUNCHED(ctx);
        NEO_CK(ctx, ctx_d2h(ctx, c_parent.data(), sh->d_mixo.p, c_parent.size() * 8));
        NEO_CK(ctx, ctx_sync(ctx));
        std::vector<K> yv((size_t)k * t * NEO_D);
        for (uint32_t i = 0; i < k; i++)
            for (uint32_t j = 0; j < t; j++)
                for (int rho = 0; rho < NEO_D; rho++) yv[((size_t)i * t + j) * NEO_D + rho] = ins[i].y[(size_t)j * d_pad + rho];
        // y vectors as [k][t][54] K = stride-2 F_q
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_mixv.p, yv.data(), yv.size() * 16, cudaMemcpyHostToDevice, ctx->stream));
        rot_mix_kernel<<<t * 2, dim3(64, 16), 0, ctx->stream>>>(sh->d_rot.p, k, sh->d_mixv.p, t, 2, sh->d_mixo.p);
        NEO_LAUNCHED(ctx);
        NEO_CK(ctx, ctx_d2h(ctx, y_parent.data(), sh->d_mixo.p, y_parent.size() * 16));
        NEO_CK(ctx, ctx_sync(ctx));
    }
    P.insert(P.end(), c_parent.begin(), c_parent.end());
    // Pi_DEC: split into k_rho planes, commit, child claims
    if ((rc = split_b_device(ctx, sh->d_mix.p, (uint64_t)NEO_D * m, sh->k_rho, sh->b, d_planes, sh->d_flags.p))) return rc;
    if ((rc = launch_commit(ctx, d_planes, sh->k_rho, m, sh->d_commits.p, TC_DIGITS_SMALL))) return rc;  // planes in {-1, 0, 1}
    {  // children's y at r: the planes are ternary
        bool done = false;
        if ((rc = launch_zrows(ctx, d_planes, sh->k_rho * NEO_D, m, t, d_vj, sh->d_ychild.p, &done))) return rc;
        if (!done) {
            child_y_kernel<<<sh->k_rho * NEO_D, 256, 0, ctx->stream>>>(d_planes, m, t, d_vj, sh->d_ychild.p);
            NEO_LAUNCHED(ctx);
        }
    }
    uint32_t flags[2];
    std::vector<uint64_t> cc((size_t)sh->k_rho * kappa * NEO_D);
    std::vector<K> yc((size_t)sh->k_rho * t * NEO_D);
    std::vector<int8_t> Xc((size_t)sh->k_rho * NEO_D * sh->m_in);
    NEO_CK(ctx, ctx_d2h(ctx, flags, sh->d_flags.p, 8));
    NEO_CK(ctx, ctx_d2h(ctx, cc.data(), sh->d_commits.p, cc.size() * 8));
    NEO_CK(ctx, ctx_d2h(ctx, yc.data(), sh->d_ychild.p, yc.size() * 16));
    NEO_CK(ctx, cudaMemcpy2DAsync(Xc.data(), sh->m_in, d_planes, m, sh->m_in, (size_t)sh->k_rho * NEO_D,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, ctx_sync(ctx));
    if ((rc = check_device_error(ctx))) return rc;
    if (flags[0]) return ctx->fail(NEO_ERR_INVARIANT, "DEC split: Z_mix entry out of range for k_rho digits");
    std::vector<K> by, bsc;
    if (nb) {
        if ((rc = upload_point(sh, r))) return rc;
        if ((rc = bus_openings(sh, d_planes, sh->k_rho, by, bsc))) return rc;
    }
    // DEC public checks (dec_children_with_commit_cached): c and core y recompose in base b
    {
        std::vector<uint64_t> cs(c_parent.size(), 0);
        uint64_t pw = 1;
        for (uint32_t i = 0; i < sh->k_rho; i++) {
            for (size_t q = 0; q < cs.size(); q++) cs[q] = gl::add(cs[q], gl::mul(cc[(size_t)i * kappa * NEO_D + q], pw));
            pw = gl::mul(pw, sh->b);
        }
        if (cs != c_parent) return ctx->fail(NEO_ERR_INVARIANT, "DEC public check failed (c)");
        std::vector<K> ysum(y_parent.size(), gl::kzero());
        pw = 1;
        for (uint32_t i = 0; i < sh->k_rho; i++) {
            for (size_t q = 0; q < ysum.size(); q++) ysum[q] = gl::kadd(ysum[q], gl::kscale(yc[(size_t)i * t * NEO_D + q], pw));
            pw = gl::mul(pw, sh->b);
        }
        for (size_t q = 0; q < ysum.size(); q++)
            if (!keq(ysum[q], y_parent[q])) return ctx->fail(NEO_ERR_INVARIANT, "DEC public check failed (y)");
    }
    children.assign(sh->k_rho, MeInst());
    uint64_t pwb[NEO_D];
    pwb[0] = 1;
    for (int q = 1; q < NEO_D; q++) pwb[q] = gl::mul(pwb[q - 1], sh->b);
    for (uint32_t i = 0; i < sh->k_rho; i++) {
        MeInst& ch = children[i];
        ch.c.assign(cc.begin() + (size_t)i * kappa * NEO_D, cc.begin() + (size_t)(i + 1) * kappa * NEO_D);
        ch.X.resize((size_t)NEO_D * sh->m_in);
        for (size_t q = 0; q < ch.X.size(); q++) ch.X[q] = gl::from_i64(Xc[(size_t)i * NEO_D * sh->m_in + q]);
        ch.r = r;
        ch.m_in = sh->m_in;
        ch.y.assign((size_t)(t + nb) * d_pad, gl::kzero());
        ch.ysc.resize(t + nb);
        for (uint32_t j = 0; j < t; j++) {
            K s = gl::kzero();
            for (int rho = 0; rho < NEO_D; rho++) {
                K v = yc[((size_t)i * t + j) * NEO_D + rho];
                ch.y[j * d_pad + rho] = v;
                s = gl::kadd(s, gl::kscale(v, pwb[rho]));
            }
            ch.ysc[j] = s;
        }
        for (uint32_t c = 0; c < nb; c++) {
            for (int rho = 0; rho < NEO_D; rho++) ch.y[(size_t)(t + c) * d_pad + rho] = by[((size_t)i * nb + c) * NEO_D + rho];
            ch.ysc[t + c] = bsc[(size_t)i * nb + c];
        }
        memcpy(ch.digest, digest, 32);
        P.insert(P.end(), ch.c.begin(), ch.c.end());
        for (uint32_t j = 0; j < t; j++)
            for (int rho = 0; rho < NEO_D; rho++) push_k(P, ch.y[j * d_pad + rho]);
        for (uint32_t c = 0; c < nb; c++)
            for (int rho = 0; rho < NEO_D; rho++) push_k(P, ch.y[(size_t)(t + c) * d_pad + rho]);
    }
    if (rec) {
        // the RLC parent: c from the mix; X, y and y_scalars recomposed from the
        // children (sum_i b^i child_i, exact: DEC splits the parent's digits)
        rec->present = true;
        rec->rhos = rhos;
        rec->children = children;
        MeInst& pa = rec->parent;
        pa = MeInst();
        pa.c = c_parent;
        pa.m_in = sh->m_in;
        pa.r = r;
        memcpy(pa.digest, digest, 32);
        pa.X.assign((size_t)NEO_D * sh->m_in, 0);
        pa.y.assign((size_t)(t + nb) * d_pad, gl::kzero());
        pa.ysc.assign(t + nb, gl::kzero());
        uint64_t pw = 1;
        for (uint32_t i = 0; i < sh->k_rho; i++) {
            const MeInst& ch = children[i];
            for (size_t q = 0; q < pa.X.size(); q++) pa.X[q] = gl::add(pa.X[q], gl::mul(ch.X[q], pw));
            for (size_t q = 0; q < pa.y.size(); q++) pa.y[q] = gl::kadd(pa.y[q], gl::kscale(ch.y[q], pw));
            for (size_t q = 0; q < pa.ysc.size(); q++) pa.ysc[q] = gl::kadd(pa.ysc[q], gl::kscale(ch.ysc[q], pw));
            pw = gl::mul(pw, sh->b);
        }
    }
    return NEO_OK;
}

}  // namespace

static int fold_step_impl(neo_gpu_shard* sh, const uint64_t* z_host, const uint64_t* d_z_in) {
    neo_gpu_ctx* ctx = sh->ctx;
    neo::Transcript& tr = *sh->tr;
    const uint64_t m = sh->m;
    const uint32_t kappa = sh->kappa, t = sh->t, ell_n = sh->ell_n, ell_d = sh->ell_d, d_sc = sh->d_sc;
    const uint32_t idx = sh->step_idx;
    const uint32_t n_acc = (uint32_t)sh->acc.size();
    const uint32_t k = 1 + n_acc;
    const uint32_t d_pad = 1u << ell_d;
    const uint32_t nb = sh->bus_cols;
    const uint64_t L = 1ULL << ell_n;
    const bool has_mem = nb > 0;
    std::vector<uint64_t>& P = sh->proof;
    P.clear();
    StepRecord& rec = sh->rec;
    rec = StepRecord();
    int rc;
    const auto t_step = hclock::now();
    NvtxStep nv;
    nv.push("fold_step");
    nv.push("witness");
    const uint64_t perms0 = tr.permutations();
    for (double& v : sh->stats) v = 0;
    auto t_ph = hclock::now();
    double mem_ms = 0;

    // ---- witness build: z -> Z (decomp) -> c = commit(Z)  (session.rs:977-978) ----
    const uint64_t* d_z = d_z_in;
    if (z_host) {
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_z.p, z_host, m * 8, cudaMemcpyHostToDevice, ctx->stream));
        d_z = sh->d_z.p;
    }
    decomp_b2_kernel<<<ceil_div(m, 256), 256, 0, ctx->stream>>>(d_z, m, sh->Zall.p);
    NEO_LAUNCHED(ctx);
    if ((rc = launch_commit(ctx, sh->Zall.p, 1, m, sh->d_commits.p, TC_DIGITS_SMALL))) return rc;  // digits in {-1, 0, 1}
    if (has_mem) {
        bus_decode_kernel<<<ceil_div((uint64_t)nb * L, 256), 256, 0, ctx->stream>>>(d_z, sh->m_in, sh->bus_base, sh->steps,
                                                                                    nb, L, sh->d_cols.p);
        NEO_LAUNCHED(ctx);
    }
    MeInst mcs;
    mcs.c.resize((size_t)kappa * NEO_D);
    std::vector<uint64_t> x(sh->m_in);
    std::vector<int8_t> Xd((size_t)NEO_D * sh->m_in);
    NEO_CK(ctx, ctx_d2h(ctx, mcs.c.data(), sh->d_commits.p, mcs.c.size() * 8));
    NEO_CK(ctx, ctx_d2h(ctx, x.data(), d_z, sh->m_in * 8));
    NEO_CK(ctx, cudaMemcpy2DAsync(Xd.data(), sh->m_in, sh->Zall.p, m, sh->m_in, NEO_D, cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, ctx_sync(ctx));
    if ((rc = check_device_error(ctx))) return rc;
    for (auto& v : x) v = gl::canon(v);
    mcs.m_in = sh->m_in;
    mcs.X.resize(Xd.size());
    for (size_t i = 0; i < Xd.size(); i++) mcs.X[i] = gl::from_i64(Xd[i]);
    P.insert(P.end(), mcs.c.begin(), mcs.c.end());
    sh->stats[1] = ms_since(t_ph);
    nv.next("bind");
    t_ph = hclock::now();

    // ---- absorb_step_memory_witness (memory_sidecar/memory.rs:86-124) ----
    {
        auto u = [&](const char* label, uint64_t v) {
            auto b8 = le64(v);
            tr.append_message(label, b8.data(), 8);
        };
        tr.append_message("step/absorb_memory_start", nullptr, 0);
        u("step/lut_count", sh->shout.size());
        for (size_t i = 0; i < sh->shout.size(); i++) {
            const ShoutInst& s = *sh->shout[i];
            u("step/lut_idx", i);
            u("shout/k", s.k);
            u("shout/d", s.d);
            u("shout/n_side", s.n_side);
            u("shout/steps", sh->steps);
            u("shout/ell", s.ell);
            tr.append_message("shout/table_digest", s.digest, 32);
        }
        u("step/mem_count", sh->twist.size());
        for (size_t i = 0; i < sh->twist.size(); i++) {
            const TwistInst& w = *sh->twist[i];
            u("step/mem_idx", i);
            u("twist/k", w.k);
            u("twist/d", w.d);
            u("twist/n_side", w.n_side);
            u("twist/steps", sh->steps);
            u("twist/ell", w.ell);
            tr.append_message("twist/init_digest", w.digest, 32);
        }
        tr.append_message("step/absorb_memory_done", nullptr, 0);
    }
    // ---- bind_header_and_instances_with_digest (engines/utils.rs:83-136) ----
    tr.append_message("phase/pi-ccs", nullptr, 0);
    tr.append_message("neo/ccs/header/v1", nullptr, 0);
    {
        uint64_t hdr[6] = {64, 2, sh->lambda, (uint64_t)(ell_n + ell_d), d_sc, (uint64_t)std::llabs(sh->slack_bits)};
        tr.append_u64s("ccs/header", hdr, 6);
        uint8_t sign = sh->slack_bits >= 0 ? 1 : 0;
        tr.append_message("ccs/slack_sign", &sign, 1);
        tr.append_message("neo/ccs/instances", nullptr, 0);
        uint64_t dims[3] = {sh->n, sh->m, t};
        tr.append_u64s("dims", dims, 3);
        for (int i = 0; i < 4; i++) tr.append_fields("mat_digest", &sh->mat_digest[i], 1);
        // absorb_sparse_polynomial (utils.rs:334-347): terms sorted by exps
        tr.append_message("neo/ccs/poly", nullptr, 0);
        uint64_t ar = t, nt = sh->ccs.n_terms;
        tr.append_u64s("arity", &ar, 1);
        tr.append_u64s("terms_len", &nt, 1);
        std::vector<uint32_t> order(nt);
        for (uint32_t i = 0; i < nt; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t bb) {
            return std::lexicographical_compare(sh->ccs.f_exps.begin() + a * t, sh->ccs.f_exps.begin() + (a + 1) * t,
                                                sh->ccs.f_exps.begin() + bb * t, sh->ccs.f_exps.begin() + (bb + 1) * t);
        });
        for (uint32_t i : order) {
            tr.append_fields("coeff", &sh->ccs.f_coeff[i], 1);
            std::vector<uint64_t> ex(sh->ccs.f_exps.begin() + i * t, sh->ccs.f_exps.begin() + (i + 1) * t);
            tr.append_u64s("exps", ex.data(), t);
        }
        tr.append_fields("x", x.data(), x.size());
        uint64_t mi = sh->m_in;
        tr.append_u64s("m_in", &mi, 1);
        tr.append_fields("c_data", mcs.c.data(), mcs.c.size());
    }
    // ---- bind_me_inputs (utils.rs:139-181) ----
    {
        tr.append_message("neo/ccs/me_inputs/v2", nullptr, 0);
        uint64_t cnt = n_acc;
        tr.append_u64s("me_count", &cnt, 1);
        for (auto& me : sh->acc) {
            tr.append_fields("c_data_in", me.c.data(), me.c.size());
            uint64_t mi = me.m_in;
            tr.append_u64s("m_in_in", &mi, 1);
            auto rf = k_flat(me.r);
            tr.append_fields("r_in", rf.data(), rf.size());
            auto yf = k_flat(me.y);
            tr.append_fields("y_elem", yf.data(), yf.size());
        }
    }
    // ---- sample_challenges (utils.rs:184-212) ----
    tr.append_message("neo/ccs/chals/v1", nullptr, 0);
    auto chal_k = [&]() {
        uint64_t c[2];
        tr.challenge_fields("chal/k", 2, c);
        return gl::kmk(c[0], c[1]);
    };
    std::vector<K> alpha(ell_d), beta(ell_d + ell_n);
    for (auto& a : alpha) a = chal_k();
    for (auto& bb : beta) bb = chal_k();
    K gamma = chal_k();
    std::vector<K> beta_a(beta.begin(), beta.begin() + ell_d), beta_r(beta.begin() + ell_d, beta.end());
    // ---- claimed_initial_sum_from_inputs (optimized_engine/common.rs:839-947), core rows ----
    K T = gl::kzero();
    if (k >= 2) {
        std::vector<K> chi_a(d_pad);
        for (uint32_t rho = 0; rho < d_pad; rho++) {
            K w = gl::kone();
            for (uint32_t bit = 0; bit < ell_d; bit++)
                w = gl::kmul(w, ((rho >> bit) & 1) ? alpha[bit] : gl::ksub(gl::kone(), alpha[bit]));
            chi_a[rho] = w;
        }
        K gk = gl::kone();
        for (uint32_t i = 0; i < k; i++) gk = gl::kmul(gk, gamma);
        K inner = gl::kzero(), gkj = gl::kone();
        for (uint32_t j = 0; j < t; j++) {
            K gi = gl::kone();
            for (uint32_t a = 0; a < n_acc; a++) {
                gi = gl::kmul(gi, gamma);  // gamma^(i-1), i = a + 2
                K ye = gl::kzero();
                for (uint32_t rho = 0; rho < d_pad; rho++) ye = gl::kadd(ye, gl::kmul(sh->acc[a].y[j * d_pad + rho], chi_a[rho]));
                inner = gl::kadd(inner, gl::kmul(gl::kmul(gi, gkj), ye));
            }
            gkj = gl::kmul(gkj, gk);
        }
        T = gl::kmul(gk, inner);
    }
    absorb_k(tr, "sumcheck/initial_sum", T);
    push_k(P, T);
    rec.alpha = alpha;
    rec.beta_a = beta_a;
    rec.beta_r = beta_r;
    rec.gamma = gamma;
    rec.T = T;
    // ---- r_cycle = sample_ext_point (neo-memory/src/ts_common.rs:22-37) ----
    std::vector<K> r_cycle = sample_ext_point(tr, "route_a/r_cycle", "route_a/cycle/0", "route_a/cycle/1", ell_n);

    sh->stats[2] = ms_since(t_ph);
    nv.next("ccs_build");
    t_ph = hclock::now();
    // ---- Pi_CCS oracle over Zall slots 0..n_acc (workspace reused across steps) ----
    const K* rin = n_acc ? sh->acc[0].r.data() : nullptr;
    if ((rc = ccs_oracle_create_dev(ctx, &sh->ccs, sh->Zall.p, k, sh->b, alpha.data(), beta_a.data(), beta_r.data(),
                                    gamma, rin, ell_d, ell_n, d_sc, &sh->orc)))
        return rc;
    neo_gpu_ccs_oracle* orc = sh->orc;
    sh->stats[3] = ms_since(t_ph);
    nv.next("time_rounds");
    t_ph = hclock::now();

    // memory oracles are rebuilt every step into the shard's slots (device buffers kept)
    size_t mem_cur = 0, ta_cur = 0;
    auto mb = [&](neo_gpu_mem_oracle** dst, int kind, uint32_t ell, const uint64_t* rp, uint32_t A, const uint64_t* ra,
                  const uint64_t* init, uint32_t nc, const uint64_t* cols, const uint64_t* w, uint64_t* claim) -> int {
        if (mem_cur == sh->mem_slots.size()) sh->mem_slots.push_back(nullptr);
        neo_gpu_mem_oracle** sl = &sh->mem_slots[mem_cur++];
        int r = mem_oracle_build_device(ctx, kind, ell, rp, A, ra, init, nc, cols, w, claim, sl);
        *dst = *sl;
        return r;
    };
    auto tb = [&](neo_gpu_twist_addr** dst, int kind, uint32_t ell, const uint64_t* rc_, uint32_t A, uint64_t n_init,
                  const uint64_t* ia, const uint64_t* iv, const uint64_t* cols) -> int {
        if (ta_cur == sh->ta_slots.size()) sh->ta_slots.push_back(nullptr);
        neo_gpu_twist_addr** sl = &sh->ta_slots[ta_cur++];
        int r = twist_addr_build_device(ctx, kind, ell, rc_, A, n_init, ia, iv, cols, sl);
        *dst = *sl;
        return r;
    };
    std::vector<Claim> claims;
    {
        Claim c;
        c.label = "ccs/time";
        c.deg = d_sc;
        c.dyn = true;
        c.sum = T;
        c.ccs = orc;
        claims.push_back(c);
    }
    std::vector<K> r_addr_s;
    std::vector<std::vector<K>> r_addr_t(sh->twist.size());
    std::vector<K> twist_read(sh->twist.size()), twist_write(sh->twist.size());
    if (has_mem) {
        auto t_mem = hclock::now();
        if ((rc = upload_point(sh, r_cycle))) return rc;
        const K* C = sh->d_cols.p;
        // ---- Shout address pre-time (memory.rs:430-621) ----
        if (!sh->shout.empty()) {
            const uint32_t ea = sh->shout[0]->ea;
            std::vector<K> sums;
            uint64_t active = 0;
            std::vector<Claim> ac;
            for (size_t i = 0; i < sh->shout.size(); i++) {
                const ShoutInst& s = *sh->shout[i];
                const K* has = C + (size_t)(s.col0 + s.ea) * L;
                // has_any_lookup: any nonzero gate in this step's bus column
                std::vector<K> hg(sh->steps);
                NEO_CK(ctx, ctx_d2h(ctx, hg.data(), has + sh->m_in, sh->steps * sizeof(K)));
                NEO_CK(ctx, ctx_sync(ctx));
                bool any = false;
                for (auto& g : hg) any |= !gl::kiszero(g);
                if (!any) {
                    sums.push_back(gl::kzero());
                    continue;
                }
                const uint64_t Pn = 1ULL << s.ea;
                K cl;
                if ((rc = addr_weights_device(ctx, ell_n, sh->d_r.p, s.ea, has, C + (size_t)s.col0 * L, s.d_table.p,
                                              std::min<uint64_t>(s.table.size(), Pn), sh->d_w.p, &cl, &sh->addr_ws)))
                    return rc;
                // ProductRoundOracle over [table, weights] (twist_oracle.rs:1719-1722), degree 2
                NEO_CK(ctx, cudaMemcpyAsync(sh->d_asm.p, s.d_table.p, Pn * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
                NEO_CK(ctx, cudaMemcpyAsync(sh->d_asm.p + Pn, sh->d_w.p, Pn * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
                neo_gpu_mem_oracle* po = nullptr;
                if ((rc = mb(&po, NEO_MEM_PRODUCT, s.ea, nullptr, 0, nullptr, nullptr, 2,
                                                           (const uint64_t*)sh->d_asm.p, nullptr, nullptr)))
                    return rc;
                Claim c;
                c.label = "shout/addr_pre";
                c.deg = 2;
                c.sum = cl;
                c.mem = po;
                ac.push_back(c);
                sums.push_back(cl);
                active |= 1ULL << i;
            }
            auto bi = le64(idx);
            tr.append_message("shout/addr_pre_time/step_idx", bi.data(), 8);
            bind_claim_sums(tr, "shout/addr_pre_time/claimed_sums", sums,
                            std::vector<std::string>(sums.size(), "shout/addr_pre"));
            for (auto& s : sums) push_k(P, s);
            P.push_back(active);
            rec.has_shout = true;
            rec.n_lut = (uint32_t)sh->shout.size();
            rec.shout_sums = sums;
            rec.shout_active = active;
            if (active == 0) {
                tr.append_message("shout/addr_pre_time/no_sumcheck", bi.data(), 8);
                r_addr_s = sample_ext_point(tr, "shout/addr_pre_time/no_sumcheck/r_addr",
                                            "shout/addr_pre_time/no_sumcheck/r_addr/0",
                                            "shout/addr_pre_time/no_sumcheck/r_addr/1", ea);
            } else {
                std::vector<K> fin;
                if ((rc = run_batched_ds(sh, "shout/addr_pre_time", idx, ac, ea, r_addr_s, fin, P, &rec.shout_pre)))
                    return rc;
            }
            rec.shout_pre.chals = r_addr_s;
            for (auto& r : r_addr_s) push_k(P, r);
        }
        // ---- Twist address pre-time (memory.rs:232-428) ----
        for (size_t i = 0; i < sh->twist.size(); i++) {
            const TwistInst& w = *sh->twist[i];
            std::vector<uint64_t> iv(2 * w.init_val.size());
            for (size_t e = 0; e < w.init_val.size(); e++) { iv[2 * e] = w.init_val[e]; iv[2 * e + 1] = 0; }
            neo_gpu_twist_addr *ro = nullptr, *wo = nullptr;
            if ((rc = assemble(sh, C, twist_read_ids(w)))) return rc;
            if ((rc = tb(&ro, 0, ell_n, (const uint64_t*)r_cycle.data(), w.ea,
                                                       w.init_addr.size(), w.init_addr.data(), iv.data(),
                                                       (const uint64_t*)sh->d_asm.p)))
                return rc;
            if ((rc = assemble(sh, C, twist_write_ids(w)))) return rc;
            if ((rc = tb(&wo, 1, ell_n, (const uint64_t*)r_cycle.data(), w.ea,
                                                       w.init_addr.size(), w.init_addr.data(), iv.data(),
                                                       (const uint64_t*)sh->d_asm.p)))
                return rc;
            auto bi = le64(i);
            tr.append_message("twist/addr_pre_time/claim_idx", bi.data(), 8);
            std::vector<std::string> labels = {"twist/read_addr_pre", "twist/write_addr_pre"};
            bind_claim_sums(tr, "twist/addr_pre_time/claimed_sums", {gl::kzero(), gl::kzero()}, labels);
            std::vector<Claim> tc(2);
            tc[0].label = labels[0]; tc[0].deg = 2; tc[0].sum = gl::kzero(); tc[0].ta = ro;
            tc[1].label = labels[1]; tc[1].deg = 2; tc[1].sum = gl::kzero(); tc[1].ta = wo;
            std::vector<K> fin;
            rec.twist_pre.emplace_back();
            if ((rc = run_batched_ds(sh, "twist/addr_pre_time", i, tc, w.ea, r_addr_t[i], fin, P, &rec.twist_pre.back())))
                return rc;
            for (auto& r : r_addr_t[i]) push_k(P, r);
            twist_read[i] = fin[0];
            twist_write[i] = fin[1];
            push_k(P, fin[0]);
            push_k(P, fin[1]);
        }
        // ---- Route-A time oracles (memory.rs:905-1033) ----
        for (size_t i = 0; i < sh->shout.size(); i++) {
            const ShoutInst& s = *sh->shout[i];
            neo_gpu_mem_oracle *vo = nullptr, *ao = nullptr, *bo = nullptr;
            K vc{}, ac_{};
            // value: [has_lookup, val] are adjacent bus columns
            if ((rc = mb(&vo, NEO_MEM_SHOUT_VALUE, ell_n, (const uint64_t*)r_cycle.data(),
                                                       0, nullptr, nullptr, 2, (const uint64_t*)(C + (size_t)(s.col0 + s.ea) * L),
                                                       nullptr, nullptr)))
                return rc;
            std::vector<uint32_t> ids = {s.col0 + s.ea};
            for (uint32_t b = 0; b < s.ea; b++) ids.push_back(s.col0 + b);
            if ((rc = assemble(sh, C, ids))) return rc;
            if ((rc = mb(&ao, NEO_MEM_SHOUT_ADAPTER, ell_n, (const uint64_t*)r_cycle.data(),
                                                       s.ea, (const uint64_t*)r_addr_s.data(), nullptr, 1 + s.ea,
                                                       (const uint64_t*)sh->d_asm.p, nullptr, nullptr)))
                return rc;
            {  // both claims from one evaluation of round 0
                neo_gpu_mem_oracle* g2[2] = {vo, ao};
                K c2[2];
                if ((rc = mem_claims_multi(ctx, g2, 2, c2, sh->d_mpart, sh->d_round, sh->h_round))) return rc;
                vc = c2[0];
                ac_ = c2[1];
            }
            // bitness over [addr_bits..., has_lookup] (adjacent columns)
            auto bw = bitness_weights(r_cycle[0], s.ea + 1, 0x53484F5554ULL + i);
            if ((rc = mb(&bo, NEO_MEM_BITNESS, ell_n, (const uint64_t*)r_cycle.data(), 0,
                                                       nullptr, nullptr, s.ea + 1, (const uint64_t*)(C + (size_t)s.col0 * L),
                                                       (const uint64_t*)bw.data(), nullptr)))  // claim 0 by construction
                return rc;
            Claim cv, ca, cb;
            cv.label = "shout/value"; cv.deg = 3; cv.sum = vc; cv.mem = vo;
            ca.label = "shout/adapter"; ca.deg = 2 + s.ea; ca.sum = ac_; ca.mem = ao;
            cb.label = "shout/bitness"; cb.deg = 3; cb.dyn = false; cb.sum = gl::kzero(); cb.mem = bo;
            claims.push_back(cv);
            claims.push_back(ca);
            claims.push_back(cb);
        }
        for (size_t i = 0; i < sh->twist.size(); i++) {
            const TwistInst& w = *sh->twist[i];
            // eval_init_at_r_addr (neo-memory/src/mem_init.rs:133-163)
            K init_r = gl::kzero();
            for (size_t e = 0; e < w.init_addr.size(); e++) {
                K chi = gl::kone();
                for (uint32_t b = 0; b < w.ea; b++)
                    chi = gl::kmul(chi, ((w.init_addr[e] >> b) & 1) ? r_addr_t[i][b] : gl::ksub(gl::kone(), r_addr_t[i][b]));
                init_r = gl::kadd(init_r, gl::kscale(chi, w.init_val[e]));
            }
            neo_gpu_mem_oracle *ro = nullptr, *wo = nullptr, *bo = nullptr;
            if ((rc = assemble(sh, C, twist_read_ids(w)))) return rc;
            if ((rc = mb(&ro, NEO_MEM_TWIST_READ, ell_n, (const uint64_t*)r_cycle.data(),
                                                       w.ea, (const uint64_t*)r_addr_t[i].data(), (const uint64_t*)&init_r,
                                                       4 + 2 * w.ea, (const uint64_t*)sh->d_asm.p, nullptr, nullptr)))
                return rc;
            if ((rc = assemble(sh, C, twist_write_ids(w)))) return rc;
            if ((rc = mb(&wo, NEO_MEM_TWIST_WRITE, ell_n, (const uint64_t*)r_cycle.data(),
                                                       w.ea, (const uint64_t*)r_addr_t[i].data(), (const uint64_t*)&init_r,
                                                       3 + w.ea, (const uint64_t*)sh->d_asm.p, nullptr, nullptr)))
                return rc;
            // bitness over [ra bits, wa bits, has_read, has_write] (adjacent columns)
            auto bw = bitness_weights(r_cycle[0], 2 * w.ea + 2, 0x5457495354ULL + i);
            if ((rc = mb(&bo, NEO_MEM_BITNESS, ell_n, (const uint64_t*)r_cycle.data(), 0,
                                                       nullptr, nullptr, 2 * w.ea + 2, (const uint64_t*)(C + (size_t)w.col0 * L),
                                                       (const uint64_t*)bw.data(), nullptr)))
                return rc;
            Claim cr, cw, cb;
            cr.label = "twist/read_check"; cr.deg = 3 + w.ea; cr.sum = twist_read[i]; cr.mem = ro;
            cw.label = "twist/write_check"; cw.deg = 3 + w.ea; cw.sum = twist_write[i]; cw.mem = wo;
            cb.label = "twist/bitness"; cb.deg = 3; cb.dyn = false; cb.sum = gl::kzero(); cb.mem = bo;
            claims.push_back(cr);
            claims.push_back(cw);
            claims.push_back(cb);
        }
        mem_ms += ms_since(t_mem);
    }
    // ---- bind_batched_dynamic_claims (memory_sidecar/transcript.rs:37-63) ----
    {
        auto bl = le64(claims.size());
        tr.append_message("batched/dynamic_bind/len", bl.data(), 8);
        for (size_t i = 0; i < claims.size(); i++) {
            auto bi = le64(i), bd = le64(claims[i].deg);
            tr.append_message("batched/dynamic_bind/claim_label", claims[i].label);
            tr.append_message("batched/dynamic_bind/claim_idx", bi.data(), 8);
            tr.append_message("batched/dynamic_bind/degree_bound", bd.data(), 8);
            uint8_t dy = claims[i].dyn ? 1 : 0;
            tr.append_message("batched/dynamic_bind/is_dynamic", &dy, 1);
            if (claims[i].dyn) absorb_k(tr, "batched/dynamic_bind/claimed_sum", claims[i].sum);
        }
    }
    // ---- batched time sum-check (route_a_time.rs:28-152) ----
    std::vector<K> r_time, finals;
    if ((rc = run_batched_ds(sh, "shard/batched_time", idx, claims, ell_n, r_time, finals, P, &rec.time))) return rc;
    K running = finals[0];
    sh->stats[4] = ms_since(t_ph);
    nv.next("ajtai_rounds");
    t_ph = hclock::now();
    // ---- Ajtai rounds: run_sumcheck_prover_ds("ccs/ajtai") ----
    auto bidx = le64(idx);
    std::vector<K> xs(d_sc + 1), ys(d_sc + 1), co;
    for (uint32_t i = 0; i <= d_sc; i++) xs[i] = gl::kfq(i);
    tr.append_message("sc/domain", "ccs/ajtai");
    tr.append_message("sc/inst_idx", bidx.data(), 8);
    absorb_k(tr, "sc/claimed_sum", running);
    for (uint32_t rd = 0; rd < ell_d; rd++) {
        if ((rc = neo_gpu_ccs_oracle_evals(orc, (const uint64_t*)xs.data(), d_sc + 1, (uint64_t*)ys.data()))) return rc;
        if (!keq(gl::kadd(ys[0], ys[1]), running))
            return ctx->fail(NEO_ERR_INVARIANT, "Ajtai sum-check: p(0)+p(1) != running sum");
        interpolate(xs, ys, co);
        for (auto& c : co) absorb_k(tr, "sumcheck/round/coeff", c);
        uint64_t c0 = tr.challenge_field("sumcheck/challenge/0");
        uint64_t c1 = tr.challenge_field("sumcheck/challenge/1");
        K r = gl::kmk(c0, c1);
        running = poly_eval(co, r);
        if ((rc = neo_gpu_ccs_oracle_fold(orc, (const uint64_t*)&r))) return rc;
        for (auto& c : co) push_k(P, c);
        rec.ajtai_polys.push_back(co);
        rec.ajtai_chals.push_back(r);
    }
    tr.append_message("sc/domain_end", "ccs/ajtai");
    tr.append_message("sc/inst_idx_end", bidx.data(), 8);
    push_k(P, running);
    rec.final_sum = running;
    uint8_t fold_digest[32];
    tr.digest32(fold_digest);

    sh->stats[5] = ms_since(t_ph);
    nv.next("me_outputs");
    t_ph = hclock::now();
    // ---- ME outputs (oracle.rs:1955-2072) + bus openings at r_time (cpu_bus.rs:195-320) ----
    std::vector<K> y_eval((size_t)k * t * NEO_D), y_sc((size_t)k * t);
    if ((rc = neo_gpu_ccs_oracle_me_outputs(orc, (uint64_t*)y_eval.data(), (uint64_t*)y_sc.data()))) return rc;
    std::vector<K> by, bsc;
    if (has_mem) {
        if ((rc = upload_point(sh, r_time))) return rc;
        if ((rc = bus_openings(sh, sh->Zall.p, k, by, bsc))) return rc;
    }
    std::vector<MeInst> outs(k);
    for (uint32_t i = 0; i < k; i++) {
        MeInst& o = outs[i];
        const MeInst& src = i == 0 ? mcs : sh->acc[i - 1];
        o.c = src.c;
        o.X = src.X;
        o.m_in = src.m_in;
        o.r = r_time;
        o.y.assign((size_t)(t + nb) * d_pad, gl::kzero());
        o.ysc.assign(t + nb, gl::kzero());
        for (uint32_t j = 0; j < t; j++) {
            for (int rho = 0; rho < NEO_D; rho++) o.y[j * d_pad + rho] = y_eval[((size_t)i * t + j) * NEO_D + rho];
            o.ysc[j] = y_sc[(size_t)i * t + j];
        }
        for (uint32_t c = 0; c < nb; c++) {
            for (int rho = 0; rho < NEO_D; rho++) o.y[(size_t)(t + c) * d_pad + rho] = by[((size_t)i * nb + c) * NEO_D + rho];
            o.ysc[t + c] = bsc[(size_t)i * nb + c];
        }
        memcpy(o.digest, fold_digest, 32);
    }
    rec.ccs_out = outs;
    for (auto& v : y_eval) push_k(P, v);
    for (auto& v : y_sc) push_k(P, v);
    for (uint32_t i = 0; i < k && nb; i++) {
        for (uint32_t c = 0; c < nb; c++)
            for (int rho = 0; rho < NEO_D; rho++) push_k(P, outs[i].y[(size_t)(t + c) * d_pad + rho]);
        for (uint32_t c = 0; c < nb; c++) push_k(P, outs[i].ysc[t + c]);
    }
    sh->stats[6] = ms_since(t_ph);
    nv.next("rlc_dec");
    t_ph = hclock::now();

    // ---- finalize_route_a_memory_prover (memory.rs:1284-1670): Twist val-eval batch + CPU ME claims at r_val ----
    std::vector<MeInst> val_claims;
    std::vector<K> r_val;
    uint8_t vdigest[32] = {0};
    if (!sh->twist.empty()) {
        auto t_mem = hclock::now();
        const K* C = sh->d_cols.p;
        std::vector<Claim> vcl;
        std::vector<uint8_t> tags;
        for (size_t i = 0; i < sh->twist.size(); i++) {
            const TwistInst& w = *sh->twist[i];
            neo_gpu_mem_oracle *lo = nullptr, *to = nullptr, *po = nullptr;
            K lc{}, tc_{}, pc{};  // set below from one evaluation of the batch's round 0
            if ((rc = assemble(sh, C, twist_val_ids(w)))) return rc;
            if ((rc = mb(&lo, NEO_MEM_VAL_EVAL, ell_n, (const uint64_t*)r_time.data(), w.ea,
                                                       (const uint64_t*)r_addr_t[i].data(), nullptr, 2 + w.ea,
                                                       (const uint64_t*)sh->d_asm.p, nullptr, nullptr)))
                return rc;
            if ((rc = mb(&to, NEO_MEM_TOTAL_INC, ell_n, nullptr, w.ea,
                                                       (const uint64_t*)r_addr_t[i].data(), nullptr, 2 + w.ea,
                                                       (const uint64_t*)sh->d_asm.p, nullptr, nullptr)))
                return rc;
            Claim c1, c2;
            c1.label = "twist/val_eval_lt"; c1.deg = w.ea + 3; c1.sum = lc; c1.mem = lo;
            c2.label = "twist/val_eval_total"; c2.deg = w.ea + 2; c2.sum = tc_; c2.mem = to;
            vcl.push_back(c1); tags.push_back(0);
            vcl.push_back(c2); tags.push_back(1);
            if (sh->has_prev) {
                if ((rc = assemble(sh, sh->d_prev_cols.p, twist_val_ids(w)))) return rc;
                if ((rc = mb(&po, NEO_MEM_TOTAL_INC, ell_n, nullptr, w.ea,
                                                           (const uint64_t*)r_addr_t[i].data(), nullptr, 2 + w.ea,
                                                           (const uint64_t*)sh->d_asm.p, nullptr, nullptr)))
                    return rc;
                Claim c3;
                c3.label = "twist/rollover_prev_total"; c3.deg = w.ea + 2; c3.sum = pc; c3.mem = po;
                vcl.push_back(c3); tags.push_back(2);
            }
        }
        {  // every val-eval claim from one evaluation of round 0
            std::vector<neo_gpu_mem_oracle*> vos;
            for (auto& c : vcl) vos.push_back(c.mem);
            std::vector<K> vs(vos.size());
            for (size_t i0 = 0; i0 < vos.size(); i0 += 24) {
                const int nn = (int)std::min<size_t>(24, vos.size() - i0);
                if ((rc = mem_claims_multi(ctx, vos.data() + i0, nn, vs.data() + i0, sh->d_mpart, sh->d_round,
                                           sh->h_round)))
                    return rc;
            }
            for (size_t i = 0; i < vcl.size(); i++) vcl[i].sum = vs[i];
        }
        auto bn = le64(sh->twist.size());
        tr.append_message("twist/val_eval/batch_start", bn.data(), 8);
        tr.append_message("twist/val_eval/step_idx", bidx.data(), 8);
        // bind_twist_val_eval_claim_sums (memory_sidecar/transcript.rs:28-35)
        auto bl = le64(vcl.size());
        tr.append_message("twist/val_eval/claimed_sums_len", bl.data(), 8);
        for (size_t i = 0; i < vcl.size(); i++) {
            auto bi = le64(i);
            tr.append_message("twist/val_eval/claim_idx", bi.data(), 8);
            tr.append_message("twist/val_eval/claim_kind", &tags[i], 1);
            absorb_k(tr, "twist/val_eval/claimed_sum", vcl[i].sum);
            push_k(P, vcl[i].sum);
        }
        std::vector<K> fin;
        rec.has_val_eval = true;
        rec.val_has_prev = sh->has_prev;
        if ((rc = run_batched_ds(sh, "twist/val_eval_batch", idx, vcl, ell_n, r_val, fin, P, &rec.val_eval))) return rc;
        tr.append_message("twist/val_eval/batch_done", nullptr, 0);
        for (auto& r : r_val) push_k(P, r);
        // emit_me_claims_for_mats (neo-memory/src/ts_common.rs:100-258): fold digest of the fork
        {
            neo::Transcript fork = tr;
            fork.append_message("fork", "cpu_bus/me_digest_val");
            fork.digest32(vdigest);
        }
        // witnesses: this step's MCS digits (and the previous step's) in valwit slots 0 (and 1)
        NEO_CK(ctx, cudaMemcpyAsync(sh->valwit.p, sh->Zall.p, (size_t)NEO_D * m, cudaMemcpyDeviceToDevice, ctx->stream));
        const uint32_t nv = sh->has_prev ? 2 : 1;
        if ((rc = upload_point(sh, r_val))) return rc;
        if ((rc = launch_chi_table(ctx, sh->d_r.p, ell_n, sh->d_chi.p))) return rc;
        if ((rc = launch_me_y(ctx, sh->ccs, sh->valwit.p, nv, m, sh->d_chi.p, ell_n, sh->b, sh->d_vj.p, sh->d_yv.p,
                              sh->d_yvsc.p, true)))
            return rc;
        std::vector<K> yv((size_t)nv * t * NEO_D), yvsc((size_t)nv * t);
        NEO_CK(ctx, ctx_d2h(ctx, yv.data(), sh->d_yv.p, yv.size() * sizeof(K)));
        NEO_CK(ctx, ctx_d2h(ctx, yvsc.data(), sh->d_yvsc.p, yvsc.size() * sizeof(K)));
        NEO_CK(ctx, ctx_sync(ctx));
        std::vector<K> vby, vbsc;
        if ((rc = bus_openings(sh, sh->valwit.p, nv, vby, vbsc))) return rc;
        for (uint32_t v = 0; v < nv; v++) {
            MeInst me;
            me.c = v == 0 ? mcs.c : sh->prev_c;
            me.X = v == 0 ? mcs.X : sh->prev_X;
            me.m_in = sh->m_in;
            me.r = r_val;
            me.y.assign((size_t)(t + nb) * d_pad, gl::kzero());
            me.ysc.assign(t + nb, gl::kzero());
            for (uint32_t j = 0; j < t; j++) {
                for (int rho = 0; rho < NEO_D; rho++) me.y[j * d_pad + rho] = yv[((size_t)v * t + j) * NEO_D + rho];
                me.ysc[j] = yvsc[(size_t)v * t + j];
            }
            for (uint32_t c = 0; c < nb; c++) {
                for (int rho = 0; rho < NEO_D; rho++) me.y[(size_t)(t + c) * d_pad + rho] = vby[((size_t)v * nb + c) * NEO_D + rho];
                me.ysc[t + c] = vbsc[(size_t)v * nb + c];
            }
            memcpy(me.digest, vdigest, 32);
            for (uint32_t j = 0; j < t + nb; j++)
                for (int rho = 0; rho < NEO_D; rho++) push_k(P, me.y[(size_t)j * d_pad + rho]);
            for (auto& s : me.ysc) push_k(P, s);
            val_claims.push_back(std::move(me));
        }
        rec.cpu_me_val = val_claims;
        mem_ms += ms_since(t_mem);
    }

    // ---- Pi_RLC + Pi_DEC, main lane (children into Zall slots 1..k_rho) ----
    const K* vj = nullptr;
    if ((rc = ccs_oracle_dev_vj(orc, &vj))) return rc;
    std::vector<MeInst> children;
    if ((rc = rlc_dec_lane(sh, "main", idx, outs, sh->Zall.p, sh->Zall.p + (size_t)NEO_D * m, r_time, vj, fold_digest,
                           children, P, &rec.main)))
        return rc;
    sh->stats[7] = ms_since(t_ph);
    nv.next("val_lane");
    t_ph = hclock::now();
    // ---- val lane (shard.rs:2195-2252) ----
    if (!val_claims.empty()) {
        tr.append_message("fold/val_lane_start", bidx.data(), 8);
        // v_j = M_j^T chi(r_val) is still in d_vj from the CPU ME claims
        std::vector<MeInst> vch;
        if ((rc = rlc_dec_lane(sh, "val", idx, val_claims, sh->valwit.p, sh->valplanes.p, r_val, sh->d_vj.p, vdigest, vch,
                               P, &rec.val)))
            return rc;
        sh->val_obligations += vch.size();
    }
    tr.append_message("fold/step_done", bidx.data(), 8);
    sh->acc.swap(children);
    if (!sh->twist.empty()) {
        // this step becomes the rollover source of the next one
        NEO_CK(ctx, cudaMemcpyAsync(sh->valwit.p + (size_t)NEO_D * m, sh->valwit.p, (size_t)NEO_D * m,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_prev_cols.p, sh->d_cols.p, (size_t)nb * L * sizeof(K), cudaMemcpyDeviceToDevice,
                                    ctx->stream));
        NEO_CK(ctx, ctx_sync(ctx));
        sh->prev_c = mcs.c;
        sh->prev_X = mcs.X;
        sh->has_prev = true;
    }
    sh->step_idx++;
    rec.valid = true;
    sh->stats[8] = ms_since(t_ph);
    nv.pop();
    sh->stats[10] = mem_ms;
    sh->stats[0] = ms_since(t_step);
    sh->stats[9] = (double)(tr.permutations() - perms0);
    return NEO_OK;
}

static int neo_gpu_shard_fold_step_impl_abi(neo_gpu_shard* sh, const uint64_t* z, uint64_t* proof, uint64_t proof_cap,
                                       uint64_t* proof_len) {
    if (!sh) return NEO_ERR_ARG;
    if (!z) return sh->ctx->fail(NEO_ERR_ARG, "fold_step: null witness");
    cudaSetDevice(sh->ctx->device);
    int rc = fold_step_impl(sh, z, nullptr);
    if (rc) return rc;
    if (proof_len) *proof_len = sh->proof.size();
    if (proof) {
        if (proof_cap < sh->proof.size()) return sh->ctx->fail(NEO_ERR_ARG, "fold_step: proof buffer too small");
        memcpy(proof, sh->proof.data(), sh->proof.size() * 8);
    }
    return NEO_OK;
}
extern "C" int neo_gpu_shard_fold_step(neo_gpu_shard* sh, const uint64_t* z, uint64_t* proof, uint64_t proof_cap,
                                       uint64_t* proof_len) { NEO_ABI_GUARD(neo_gpu_shard_fold_step_impl_abi(sh, z, proof, proof_cap, proof_len)) }

// Variant with the step witness already resident on the device (d_z: m words).
static int neo_gpu_shard_fold_step_device_impl_abi(neo_gpu_shard* sh, const uint64_t* d_z, uint64_t* proof_len) {
    if (!sh) return NEO_ERR_ARG;
    if (!d_z) return sh->ctx->fail(NEO_ERR_ARG, "fold_step_device: null witness");
    cudaSetDevice(sh->ctx->device);
    int rc = fold_step_impl(sh, nullptr, d_z);
    if (rc) return rc;
    if (proof_len) *proof_len = sh->proof.size();
    return NEO_OK;
}
extern "C" int neo_gpu_shard_fold_step_device(neo_gpu_shard* sh, const uint64_t* d_z, uint64_t* proof_len) { NEO_ABI_GUARD(neo_gpu_shard_fold_step_device_impl_abi(sh, d_z, proof_len)) }

// ---------------------------------------------------------------------------
// Trace chunk -> witness on the device (R1csCpu::build_ccs_chunks with the
// shared CPU bus, crates/neo-memory/src/cpu/r1cs_adapter.rs:372-650).
// Events arrive packed, per step j < S: Shout instance i at 3 S i words
// [has_lookup | key | val], then Twist instance i at 3 S n_shout + 6 S i
// [has_read | ra | rv | has_write | wa | wv].
namespace {

constexpr uint32_t TRACE_MAX_STEPS = 16384;  // the increment sort's keys fit shared memory
constexpr int TRACE_J_BITS = 15;

__global__ void trace_state_init_kernel(uint64_t* __restrict__ state, uint64_t n, const uint64_t* __restrict__ addr,
                                        const uint64_t* __restrict__ val) {
    const uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (e < n) state[addr[e]] = val[e];
}

// Shout bus cells of step j: address bits (least significant first), has_lookup, val
__global__ void trace_shout_bus_kernel(uint64_t* __restrict__ z, uint64_t bus_base, uint64_t cap, uint64_t S,
                                       uint32_t col0, uint32_t ea, const uint64_t* __restrict__ ev) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j >= S || !ev[j]) return;
    const uint64_t key = ev[S + j];
    for (uint32_t b = 0; b < ea; b++) z[bus_base + (uint64_t)(col0 + b) * cap + j] = (key >> b) & 1;
    z[bus_base + (uint64_t)(col0 + ea) * cap + j] = 1;
    z[bus_base + (uint64_t)(col0 + ea + 1) * cap + j] = gl::canon(ev[2 * S + j]);
}

// Twist bus cells of step j: ra bits, wa bits, has_read, has_write, wv, rv
// (the increment comes from trace_twist_inc_kernel)
__global__ void trace_twist_bus_kernel(uint64_t* __restrict__ z, uint64_t bus_base, uint64_t cap, uint64_t S,
                                       uint32_t col0, uint32_t ea, const uint64_t* __restrict__ ev) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j >= S) return;
    auto cell = [&](uint32_t col) -> uint64_t& { return z[bus_base + (uint64_t)col * cap + j]; };
    if (ev[j]) {
        const uint64_t ra = ev[S + j];
        for (uint32_t b = 0; b < ea; b++) cell(col0 + b) = (ra >> b) & 1;
        cell(col0 + 2 * ea) = 1;
        cell(col0 + 2 * ea + 3) = gl::canon(ev[2 * S + j]);
    }
    if (ev[3 * S + j]) {
        const uint64_t wa = ev[4 * S + j];
        for (uint32_t b = 0; b < ea; b++) cell(col0 + ea + b) = (wa >> b) & 1;
        cell(col0 + 2 * ea + 1) = 1;
        cell(col0 + 2 * ea + 2) = gl::canon(ev[5 * S + j]);
    }
}

// inc_at_write_addr of every write of one Twist instance and the memory after
// the chunk (one block): the writes sorted by (address, step) in shared
// memory; a write's previous value is the write before it in that order when
// it has the same address, else the memory at the chunk's start.  All reads
// of the memory happen before the barrier, the updates (the last write of
// each address) after it.
__global__ void __launch_bounds__(1024) trace_twist_inc_kernel(uint64_t* __restrict__ z, uint64_t bus_base,
                                                               uint64_t cap, uint64_t S, uint32_t n_sort,
                                                               uint32_t inc_col, const uint64_t* __restrict__ ev,
                                                               uint64_t* __restrict__ state) {
    extern __shared__ uint64_t keys[];
    const uint64_t NONE = ~0ull;
    const uint64_t* has_w = ev + 3 * S;
    const uint64_t* wa = ev + 4 * S;
    const uint64_t* wv = ev + 5 * S;
    for (uint32_t i = threadIdx.x; i < n_sort; i += blockDim.x)
        keys[i] = (i < S && has_w[i]) ? (wa[i] << TRACE_J_BITS) | i : NONE;
    __syncthreads();
    for (uint32_t k = 2; k <= n_sort; k <<= 1)  // bitonic sort, ascending
        for (uint32_t h = k >> 1; h > 0; h >>= 1) {
            for (uint32_t i = threadIdx.x; i < n_sort; i += blockDim.x) {
                const uint32_t l = i ^ h;
                if (l > i) {
                    const uint64_t a = keys[i], b = keys[l];
                    if ((a > b) == ((i & k) == 0)) {
                        keys[i] = b;
                        keys[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    const uint64_t jmask = (1ull << TRACE_J_BITS) - 1;
    for (uint32_t i = threadIdx.x; i < n_sort; i += blockDim.x) {
        const uint64_t key = keys[i];
        if (key == NONE) continue;
        const uint64_t j = key & jmask, addr = key >> TRACE_J_BITS;
        const bool same = i > 0 && keys[i - 1] != NONE && (keys[i - 1] >> TRACE_J_BITS) == addr;
        const uint64_t old = same ? gl::canon(wv[keys[i - 1] & jmask]) : state[addr];
        z[bus_base + (uint64_t)inc_col * cap + j] = gl::sub(gl::canon(wv[j]), old);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n_sort; i += blockDim.x) {
        const uint64_t key = keys[i];
        if (key == NONE) continue;
        const uint64_t addr = key >> TRACE_J_BITS;
        const bool last = i + 1 == n_sort || keys[i + 1] == NONE || (keys[i + 1] >> TRACE_J_BITS) != addr;
        if (last) state[addr] = gl::canon(wv[key & jmask]);
    }
}

}  // namespace

static int neo_gpu_shard_fold_step_trace_impl_abi(neo_gpu_shard* sh, const uint64_t* z_cpu, uint64_t z_cpu_len,
                                                  const neo_trace_chunk* trc, uint64_t* proof, uint64_t proof_cap,
                                                  uint64_t* proof_len) {
    if (!sh) return NEO_ERR_ARG;
    neo_gpu_ctx* ctx = sh->ctx;
    if (!trc || (z_cpu_len && !z_cpu)) return ctx->fail(NEO_ERR_ARG, "fold_step_trace: null argument");
    if (sh->steps == 0) return ctx->fail(NEO_ERR_ARG, "fold_step_trace: the shard has no memory instances");
    if (z_cpu_len > sh->bus_base) return ctx->fail(NEO_ERR_ARG, "fold_step_trace: CPU witness overlaps the bus tail");
    const uint64_t S = trc->steps;
    if (S > sh->steps || S > TRACE_MAX_STEPS) return ctx->fail(NEO_ERR_ARG, "fold_step_trace: too many steps");
    const size_t ns = sh->shout.size(), nt = sh->twist.size();
    if ((ns && !trc->shout) || (nt && !trc->twist)) return ctx->fail(NEO_ERR_ARG, "fold_step_trace: missing events");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    // validate and pack the events (the reference's build errors: bad flags,
    // Twist addresses outside the memory)
    const size_t words = (3 * ns + 6 * nt) * S;
    NEO_CK(ctx, sh->h_events.ensure(words ? words : 1));
    uint64_t* h = sh->h_events.p;
    auto flag = [](const uint8_t* f, uint64_t j, bool* ok) -> uint64_t {
        const uint8_t v = f ? f[j] : 0;
        if (v > 1) *ok = false;
        return v;
    };
    bool ok = true;
    for (size_t i = 0; i < ns && ok; i++) {
        const neo_shout_events& e = trc->shout[i];
        uint64_t* o = h + 3 * S * i;
        for (uint64_t j = 0; j < S; j++) {
            o[j] = flag(e.has_lookup, j, &ok);
            if (o[j] && (!e.key || !e.val)) ok = false;
            o[S + j] = o[j] && ok ? e.key[j] & ((1ull << sh->shout[i]->ea) - 1) : 0;
            o[2 * S + j] = o[j] && ok ? e.val[j] : 0;
        }
    }
    for (size_t i = 0; i < nt && ok; i++) {
        const neo_twist_events& e = trc->twist[i];
        const uint32_t ea = sh->twist[i]->ea;
        uint64_t* o = h + 3 * S * ns + 6 * S * i;
        for (uint64_t j = 0; j < S && ok; j++) {
            o[j] = flag(e.has_read, j, &ok);
            o[3 * S + j] = flag(e.has_write, j, &ok);
            if ((o[j] && (!e.ra || !e.rv)) || (o[3 * S + j] && (!e.wa || !e.wv))) ok = false;
            if (!ok) break;
            o[S + j] = o[j] ? e.ra[j] : 0;
            o[2 * S + j] = o[j] ? e.rv[j] : 0;
            o[4 * S + j] = o[3 * S + j] ? e.wa[j] : 0;
            o[5 * S + j] = o[3 * S + j] ? e.wv[j] : 0;
            if ((o[S + j] >> ea) || (o[4 * S + j] >> ea))
                return ctx->fail(NEO_ERR_ARG, "fold_step_trace: Twist address outside the memory");
        }
    }
    if (!ok) return ctx->fail(NEO_ERR_ARG, "fold_step_trace: malformed events (flag not 0/1 or null array)");
    // the memories at the chunk's start, rebuilt from the MemInit when stale
    for (size_t i = 0; i < nt; i++) {
        TwistInst& ti = *sh->twist[i];
        if (ti.state_valid) continue;
        const uint64_t cells = 1ull << ti.ea;
        NEO_CK(ctx, ti.d_state.ensure(cells));
        NEO_CK(ctx, cudaMemsetAsync(ti.d_state.p, 0, cells * 8, st));
        const uint64_t n = ti.init_addr.size();
        if (n) {
            DevBuf<uint64_t> da, dv;
            NEO_CK(ctx, da.alloc(n));
            NEO_CK(ctx, dv.alloc(n));
            NEO_CK(ctx, cudaMemcpyAsync(da.p, ti.init_addr.data(), n * 8, cudaMemcpyHostToDevice, st));
            NEO_CK(ctx, cudaMemcpyAsync(dv.p, ti.init_val.data(), n * 8, cudaMemcpyHostToDevice, st));
            trace_state_init_kernel<<<ceil_div(n, 256), 256, 0, st>>>(ti.d_state.p, n, da.p, dv.p);
            NEO_LAUNCHED(ctx);
            NEO_CK(ctx, ctx_sync(ctx));  // the staging buffers go out of scope
        }
        ti.state_valid = true;
    }
    // z = CPU witness, zeros, then the bus tail from the events
    const uint64_t m = sh->m;
    NEO_CK(ctx, cudaMemsetAsync(sh->d_z.p, 0, m * 8, st));
    if (z_cpu_len) NEO_CK(ctx, cudaMemcpyAsync(sh->d_z.p, z_cpu, z_cpu_len * 8, cudaMemcpyHostToDevice, st));
    if (words) {
        NEO_CK(ctx, sh->d_events.ensure(words));
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_events.p, h, words * 8, cudaMemcpyHostToDevice, st));
    }
    if (S) {
        for (size_t i = 0; i < ns; i++) {
            trace_shout_bus_kernel<<<ceil_div(S, 256), 256, 0, st>>>(sh->d_z.p, sh->bus_base, sh->steps, S,
                                                                     sh->shout[i]->col0, sh->shout[i]->ea,
                                                                     sh->d_events.p + 3 * S * i);
            NEO_LAUNCHED(ctx);
        }
        uint32_t n_sort = 1;
        while (n_sort < S) n_sort <<= 1;
        static SmemLimit inc_smem;
        NEO_CK(ctx, inc_smem.at_least(trace_twist_inc_kernel, (size_t)n_sort * 8));
        for (size_t i = 0; i < nt; i++) {
            const TwistInst& ti = *sh->twist[i];
            const uint64_t* ev = sh->d_events.p + 3 * S * ns + 6 * S * i;
            trace_twist_bus_kernel<<<ceil_div(S, 256), 256, 0, st>>>(sh->d_z.p, sh->bus_base, sh->steps, S, ti.col0,
                                                                     ti.ea, ev);
            NEO_LAUNCHED(ctx);
            trace_twist_inc_kernel<<<1, 1024, (size_t)n_sort * 8, st>>>(sh->d_z.p, sh->bus_base, sh->steps, S, n_sort,
                                                                       ti.col0 + 2 * ti.ea + 4, ev, ti.d_state.p);
            NEO_LAUNCHED(ctx);
        }
    }
    int rc = fold_step_impl(sh, nullptr, sh->d_z.p);
    if (rc) {
        for (auto& ti : sh->twist) ti->state_valid = false;  // the memory advanced; the MemInit did not
        return rc;
    }
    // the next step's MemInit: the nonzero cells of each memory, by address
    for (size_t i = 0; i < nt; i++) {
        TwistInst& ti = *sh->twist[i];
        const uint64_t cells = 1ull << ti.ea;
        std::vector<uint64_t> dense(cells), a, v;
        NEO_CK(ctx, ctx_d2h(ctx, dense.data(), ti.d_state.p, cells * 8));
        NEO_CK(ctx, ctx_sync(ctx));
        for (uint64_t c = 0; c < cells; c++)
            if (dense[c]) {
                a.push_back(c);
                v.push_back(dense[c]);
            }
        if (!twist_set_init(ti, a.size(), a.data(), v.data()))
            return ctx->fail(NEO_ERR_INVARIANT, "fold_step_trace: memory state is not a valid MemInit");
        ti.state_valid = true;
    }
    if (proof_len) *proof_len = sh->proof.size();
    if (proof) {
        if (proof_cap < sh->proof.size()) return ctx->fail(NEO_ERR_ARG, "fold_step_trace: proof buffer too small");
        memcpy(proof, sh->proof.data(), sh->proof.size() * 8);
    }
    return NEO_OK;
}
extern "C" int neo_gpu_shard_fold_step_trace(neo_gpu_shard* sh, const uint64_t* z_cpu, uint64_t z_cpu_len,
                                             const neo_trace_chunk* trace, uint64_t* proof, uint64_t proof_cap,
                                             uint64_t* proof_len) {
    NEO_ABI_GUARD(neo_gpu_shard_fold_step_trace_impl_abi(sh, z_cpu, z_cpu_len, trace, proof, proof_cap, proof_len))
}

// ---------------------------------------------------------------------------
// StepProof in struct order (crates/neo-fold/src/shard_proof_types.rs:45-131):
// a canonical word dump, every Vec prefixed by its length, K = (re, im),
// F and integers one word, [u8; 32] digests four little-endian words, byte
// strings a length then 8 bytes per word, Option a 0 / 1 word then the value.
// ---------------------------------------------------------------------------
namespace {
struct WordWriter {
    std::vector<uint64_t> w;
    void u(uint64_t v) { w.push_back(v); }
    void k(K v) {
        w.push_back(v.re);
        w.push_back(v.im);
    }
    void fvec(const std::vector<uint64_t>& v) {
        u(v.size());
        w.insert(w.end(), v.begin(), v.end());
    }
    void kvec(const std::vector<K>& v) {
        u(v.size());
        for (auto& x : v) k(x);
    }
    void digest(const uint8_t* d) {
        for (int i = 0; i < 4; i++) {
            uint64_t x = 0;
            for (int b = 0; b < 8; b++) x |= (uint64_t)d[8 * i + b] << (8 * b);
            u(x);
        }
    }
    void bytes(const std::string& s) {
        u(s.size());
        for (size_t i = 0; i < s.size(); i += 8) {
            uint64_t x = 0;
            for (size_t b = 0; b < 8 && i + b < s.size(); b++) x |= (uint64_t)(uint8_t)s[i + b] << (8 * b);
            u(x);
        }
    }
};

// MeInstance (crates/neo-ccs/src/relations.rs:234-258): c, X, r, y, y_scalars,
// m_in, fold_digest, c_step_coords (empty), u_offset, u_len (0)
void write_me(WordWriter& W, const MeInst& me, uint32_t kappa, uint32_t d_pad) {
    W.u(NEO_D);
    W.u(kappa);
    W.fvec(me.c);
    W.u(NEO_D);
    W.u(me.m_in);
    W.fvec(me.X);
    W.kvec(me.r);
    const size_t rows = me.y.size() / d_pad;
    W.u(rows);
    for (size_t r = 0; r < rows; r++) {
        W.u(d_pad);
        for (uint32_t e = 0; e < d_pad; e++) W.k(me.y[r * d_pad + e]);
    }
    W.kvec(me.ysc);
    W.u(me.m_in);
    W.digest(me.digest);
    W.u(0);
    W.u(0);
    W.u(0);
}

void write_mes(WordWriter& W, const std::vector<MeInst>& v, uint32_t kappa, uint32_t d_pad) {
    W.u(v.size());
    for (auto& me : v) write_me(W, me, kappa, d_pad);
}

// rho_i = rot(a_i): column j = cf(a_i X^j mod Phi_81) (X^54 = -X^27 - 1); the
// identity when the lane mixes one instance (common.rs:557-562)
void write_rhos(WordWriter& W, const std::vector<int8_t>& rhos, uint32_t k) {
    W.u(k);
    for (uint32_t i = 0; i < k; i++) {
        int64_t R[NEO_D][NEO_D];
        int64_t col[NEO_D];
        for (int q = 0; q < NEO_D; q++) col[q] = rhos[(size_t)i * NEO_D + q];
        for (int j = 0; j < NEO_D; j++) {
            for (int q = 0; q < NEO_D; q++) R[q][j] = k == 1 ? (q == j) : col[q];
            const int64_t last = col[NEO_D - 1];
            for (int q = NEO_D - 1; q > 0; q--) col[q] = col[q - 1];
            col[0] = -last;
            col[27] -= last;
        }
        W.u(NEO_D);
        W.u(NEO_D);
        W.u((uint64_t)NEO_D * NEO_D);
        for (int q = 0; q < NEO_D; q++)
            for (int j = 0; j < NEO_D; j++) W.u(gl::from_i64(R[q][j]));
    }
}

void write_polys(WordWriter& W, const std::vector<std::vector<std::vector<K>>>& polys) {
    W.u(polys.size());
    for (auto& claim : polys) {
        W.u(claim.size());
        for (auto& round : claim) W.kvec(round);
    }
}

void write_lane(WordWriter& W, const LaneRec& L, uint32_t kappa, uint32_t d_pad) {
    write_rhos(W, L.rhos, (uint32_t)(L.rhos.size() / NEO_D));
    write_me(W, L.parent, kappa, d_pad);
    write_mes(W, L.children, kappa, d_pad);
}
}  // namespace

static int neo_gpu_shard_step_proof_impl_abi(neo_gpu_shard* sh, uint64_t* out, uint64_t cap, uint64_t* len) {
    if (!sh || !len) return NEO_ERR_ARG;
    const StepRecord& R = sh->rec;
    if (!R.valid) return sh->ctx->fail(NEO_ERR_ARG, "step_proof: no completed fold step");
    const uint32_t kappa = sh->kappa, d_pad = 1u << sh->ell_d;
    WordWriter W;
    // fold: FoldStep
    write_mes(W, R.ccs_out, kappa, d_pad);
    W.u(R.ajtai_polys.size());  // PiCcsProof::sumcheck_rounds
    for (auto& co : R.ajtai_polys) W.kvec(co);
    W.u(1);  // sc_initial_sum: Some(T)
    W.k(R.T);
    {
        std::vector<K> ch = R.time.chals;  // sumcheck_challenges: r_time || alpha'
        ch.insert(ch.end(), R.ajtai_chals.begin(), R.ajtai_chals.end());
        W.kvec(ch);
    }
    W.kvec(R.alpha);  // challenges_public
    W.kvec(R.beta_a);
    W.kvec(R.beta_r);
    W.k(R.gamma);
    W.k(R.final_sum);  // sumcheck_final
    W.u(0);            // header_digest: empty
    W.u(0);            // _extra: None
    write_lane(W, R.main, kappa, d_pad);
    // mem: MemSidecarProof
    write_mes(W, R.cpu_me_val, kappa, d_pad);
    // shout_addr_pre: ShoutAddrPreProof, empty without Shout instances
    W.kvec(R.shout_sums);
    W.u(R.shout_active);
    write_polys(W, R.shout_pre.polys);
    W.kvec(R.has_shout ? R.shout_pre.chals : std::vector<K>());
    // proofs: Vec<MemOrLutProof>, the Shout entries first (memory.rs:1555-1569);
    // enum tags in declaration order, Twist = 0, Shout = 1
    W.u(R.n_lut + R.twist_pre.size());
    for (uint32_t i = 0; i < R.n_lut; i++) {
        W.u(1);  // ShoutProof { addr_pre: BatchedAddrProof::default() }
        W.u(0);
        W.u(0);
        W.u(0);
    }
    const uint32_t per_mem = R.val_has_prev ? 3 : 2;
    for (size_t i = 0; i < R.twist_pre.size(); i++) {
        const BatchRec& tp = R.twist_pre[i];
        W.u(0);
        W.kvec(tp.sums);  // addr_pre: claimed sums (zero), read / write rounds, r_addr
        write_polys(W, tp.polys);
        W.kvec(tp.chals);
        const size_t base = per_mem * i;  // val_eval: this instance's claims of the batch
        const bool ve = R.has_val_eval && base + per_mem <= R.val_eval.sums.size();
        W.u(ve ? 1 : 0);
        if (!ve) continue;
        for (uint32_t c = 0; c < per_mem; c++) {
            if (c == 2) W.u(1);  // Some(claimed_prev_inc_sum_total)
            W.k(R.val_eval.sums[base + c]);
            if (c == 2) W.u(1);  // Some(rounds_prev_total)
            W.u(R.val_eval.polys[base + c].size());
            for (auto& rd : R.val_eval.polys[base + c]) W.kvec(rd);
        }
        if (per_mem == 2) {
            W.u(0);
            W.u(0);
        }
    }
    // batched_time: BatchedTimeProof
    W.kvec(R.time.sums);
    W.u(R.time.degs.size());
    for (auto d : R.time.degs) W.u(d);
    W.u(R.time.labels.size());
    for (auto& l : R.time.labels) W.bytes(l);
    write_polys(W, R.time.polys);
    // val_fold: Option<RlcDecProof>
    W.u(R.val.present ? 1 : 0);
    if (R.val.present) write_lane(W, R.val, kappa, d_pad);
    *len = W.w.size();
    if (!out) return NEO_OK;
    if (cap < W.w.size()) return sh->ctx->fail(NEO_ERR_ARG, "step_proof: buffer too small");
    memcpy(out, W.w.data(), W.w.size() * 8);
    return NEO_OK;
}
extern "C" int neo_gpu_shard_step_proof(neo_gpu_shard* sh, uint64_t* out, uint64_t cap, uint64_t* len) {
    NEO_ABI_GUARD(neo_gpu_shard_step_proof_impl_abi(sh, out, cap, len))
}

static int neo_gpu_shard_transcript_state_impl_abi(const neo_gpu_shard* sh, uint64_t* st8) {
    if (!sh || !st8) return NEO_ERR_ARG;
    memcpy(st8, sh->tr->state(), 64);
    return NEO_OK;
}
extern "C" int neo_gpu_shard_transcript_state(const neo_gpu_shard* sh, uint64_t* st8) { NEO_ABI_GUARD(neo_gpu_shard_transcript_state_impl_abi(sh, st8)) }

static int neo_gpu_shard_ccs_digest_impl_abi(const neo_gpu_shard* sh, uint64_t* d4) {
    if (!sh || !d4) return NEO_ERR_ARG;
    memcpy(d4, sh->mat_digest, 32);
    return NEO_OK;
}
extern "C" int neo_gpu_shard_ccs_digest(const neo_gpu_shard* sh, uint64_t* d4) { NEO_ABI_GUARD(neo_gpu_shard_ccs_digest_impl_abi(sh, d4)) }

static int neo_gpu_shard_step_stats_impl_abi(const neo_gpu_shard* sh, double* out, uint32_t n) {
    if (!sh || !out) return NEO_ERR_ARG;
    for (uint32_t i = 0; i < n && i < 12; i++) out[i] = sh->stats[i];
    return NEO_OK;
}
extern "C" int neo_gpu_shard_step_stats(const neo_gpu_shard* sh, double* out, uint32_t n) { NEO_ABI_GUARD(neo_gpu_shard_step_stats_impl_abi(sh, out, n)) }

static int neo_gpu_shard_set_twist_init_impl_abi(neo_gpu_shard* sh, uint32_t mem_idx, uint64_t n_init,
                                            const uint64_t* init_addr, const uint64_t* init_val) {
    if (!sh) return NEO_ERR_ARG;
    neo_gpu_ctx* ctx = sh->ctx;
    if (mem_idx >= sh->twist.size()) return ctx->fail(NEO_ERR_ARG, "shard_set_twist_init: mem_idx out of range");
    if (n_init && (!init_addr || !init_val)) return ctx->fail(NEO_ERR_ARG, "shard_set_twist_init: init is null");
    TwistInst tmp;
    tmp.ea = sh->twist[mem_idx]->ea;
    if (!twist_set_init(tmp, n_init, init_addr, init_val))
        return ctx->fail(NEO_ERR_ARG, "shard_set_twist_init: addresses must be strictly increasing and < 2^ell_addr");
    TwistInst& ti = *sh->twist[mem_idx];
    ti.init_addr.swap(tmp.init_addr);
    ti.init_val.swap(tmp.init_val);
    memcpy(ti.digest, tmp.digest, 32);
    ti.state_valid = false;  // a trace step rebuilds its memory from this MemInit
    return NEO_OK;
}
extern "C" int neo_gpu_shard_set_twist_init(neo_gpu_shard* sh, uint32_t mem_idx, uint64_t n_init,
                                            const uint64_t* init_addr, const uint64_t* init_val) { NEO_ABI_GUARD(neo_gpu_shard_set_twist_init_impl_abi(sh, mem_idx, n_init, init_addr, init_val)) }

static int neo_gpu_shard_val_obligations_impl_abi(const neo_gpu_shard* sh, uint64_t* count) {
    if (!sh || !count) return NEO_ERR_ARG;
    *count = sh->val_obligations;
    return NEO_OK;
}
extern "C" int neo_gpu_shard_val_obligations(const neo_gpu_shard* sh, uint64_t* count) { NEO_ABI_GUARD(neo_gpu_shard_val_obligations_impl_abi(sh, count)) }

// ------------------------------------------------------ checkpoint / resume --
// The state a shard carries from one fold step to the next, as one byte
// string: the transcript position, the step index, the accumulator (its ME
// instances on the host and its digit planes, Zall slots 1..k), the val lane's
// previous MCS witness, commitment and public input, its obligation count, the
// Twist MemInits and the previous step's decoded bus columns (the rollover
// claim).  Everything else a shard holds is either fixed at creation (CCS,
// tables, buffers) or rebuilt every step (oracle workspaces).  A serving loop
// evicts a shard's device state with it and restores it later, or resumes
// after the process is restarted; the restored shard proves the next steps
// exactly as the uninterrupted one would.
namespace {
constexpr uint64_t CKPT_MAGIC = 0x3154504B434F454EULL;  // "NEOCKPT1"
constexpr uint64_t CKPT_VERSION = 1;

// counts (dst == null) or writes the checkpoint
struct CkptWriter {
    uint8_t* dst = nullptr;
    uint64_t n = 0;
    neo_gpu_ctx* ctx = nullptr;
    void put(const void* p, uint64_t bytes) {
        if (dst && bytes) memcpy(dst + n, p, bytes);
        n += bytes;
    }
    void u64(uint64_t v) { put(&v, 8); }
    void u64s(const std::vector<uint64_t>& v) { u64(v.size()); put(v.data(), v.size() * 8); }
    void ks(const std::vector<K>& v) { u64(v.size()); put(v.data(), v.size() * sizeof(K)); }
    cudaError_t dev(const void* dptr, uint64_t bytes) {
        u64(bytes);
        cudaError_t e = cudaSuccess;
        if (dst && bytes) e = cudaMemcpyAsync(dst + n, dptr, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        n += bytes;
        return e;
    }
};

struct CkptReader {
    const uint8_t* p;
    uint64_t left;
    bool ok = true;
    bool get(void* dst, uint64_t bytes) {
        if (!ok || bytes > left) return ok = false;
        if (bytes) memcpy(dst, p, bytes);
        p += bytes;
        left -= bytes;
        return true;
    }
    uint64_t u64() {
        uint64_t v = 0;
        get(&v, 8);
        return v;
    }
    template <typename T>
    void vec(std::vector<T>& v) {
        const uint64_t n = u64();
        if (!ok || n > left / sizeof(T)) { ok = false; return; }
        v.resize(n);
        get(v.data(), n * sizeof(T));
    }
    // a device blob of exactly `bytes` (0 allowed when the shard has no such state yet)
    const uint8_t* blob(uint64_t* bytes) {
        *bytes = u64();
        if (!ok || *bytes > left) { ok = false; return nullptr; }
        const uint8_t* b = p;
        p += *bytes;
        left -= *bytes;
        return b;
    }
};

// header fields: the shard a checkpoint may be restored into
void ckpt_header(const neo_gpu_shard* sh, uint64_t h[14]) {
    h[0] = CKPT_MAGIC; h[1] = CKPT_VERSION; h[2] = sh->n; h[3] = sh->m; h[4] = sh->t; h[5] = sh->k_rho;
    h[6] = sh->kappa; h[7] = sh->bus_cols; h[8] = sh->m_in; h[9] = sh->ell_n; h[10] = sh->shout.size();
    h[11] = sh->twist.size(); h[12] = sh->steps; h[13] = sh->b;
}

int ckpt_write(neo_gpu_shard* sh, CkptWriter& w) {
    neo_gpu_ctx* ctx = sh->ctx;
    uint64_t h[14];
    ckpt_header(sh, h);
    for (uint64_t v : h) w.u64(v);
    w.put(sh->mat_digest, 32);
    uint64_t st[8], perms;
    uint32_t absorbed;
    sh->tr->save(st, &absorbed, &perms);
    w.put(st, 64);
    w.u64(absorbed);
    w.u64(perms);
    w.u64(sh->step_idx);
    w.u64(sh->has_prev ? 1 : 0);
    w.u64(sh->val_obligations);
    w.u64(sh->acc.size());
    for (const MeInst& me : sh->acc) {
        w.u64s(me.c);
        w.u64s(me.X);
        w.ks(me.r);
        w.ks(me.y);
        w.ks(me.ysc);
        w.u64(me.m_in);
        w.put(me.digest, 32);
    }
    w.u64s(sh->prev_c);
    w.u64s(sh->prev_X);
    for (auto& ti : sh->twist) {
        w.u64s(ti->init_addr);
        w.u64s(ti->init_val);
        w.put(ti->digest, 32);
    }
    const uint64_t plane = (uint64_t)NEO_D * sh->m;
    NEO_CK(ctx, w.dev(sh->Zall.p + plane, sh->acc.size() * plane));
    NEO_CK(ctx, w.dev(sh->valwit.p, sh->has_prev ? sh->valwit.bytes() : 0));
    NEO_CK(ctx, w.dev(sh->d_prev_cols.p, sh->has_prev ? sh->d_prev_cols.bytes() : 0));
    if (w.dst) NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
}  // namespace

static int neo_gpu_shard_checkpoint_impl_abi(neo_gpu_shard* sh, uint8_t* buf, uint64_t cap, uint64_t* len) {
    if (!sh || !len) return NEO_ERR_ARG;
    neo_gpu_ctx* ctx = sh->ctx;
    cudaSetDevice(ctx->device);
    CkptWriter count;
    count.ctx = ctx;
    int rc = ckpt_write(sh, count);
    if (rc) return rc;
    *len = count.n;
    if (!buf) return NEO_OK;
    if (cap < count.n) return ctx->fail(NEO_ERR_ARG, "shard_checkpoint: buffer too small (see *len)");
    NEO_CK(ctx, ctx_sync(ctx));  // the last step's device work is part of the state
    CkptWriter w;
    w.dst = buf;
    w.ctx = ctx;
    return ckpt_write(sh, w);
}
extern "C" int neo_gpu_shard_checkpoint(neo_gpu_shard* sh, uint8_t* buf, uint64_t cap, uint64_t* len) { NEO_ABI_GUARD(neo_gpu_shard_checkpoint_impl_abi(sh, buf, cap, len)) }

static int neo_gpu_shard_restore_impl_abi(neo_gpu_shard* sh, const uint8_t* buf, uint64_t len) {
    if (!sh) return NEO_ERR_ARG;
    neo_gpu_ctx* ctx = sh->ctx;
    if (!buf) return ctx->fail(NEO_ERR_ARG, "shard_restore: null buffer");
    cudaSetDevice(ctx->device);
    CkptReader r{buf, len};
    uint64_t want[14], got[14];
    ckpt_header(sh, want);
    for (auto& v : got) v = r.u64();
    uint8_t dig[32];
    r.get(dig, 32);
    if (!r.ok || memcmp(got, want, sizeof want) || memcmp(dig, sh->mat_digest, 32))
        return ctx->fail(NEO_ERR_ARG, "shard_restore: checkpoint of another shard shape, CCS or format");
    uint64_t st[8];
    r.get(st, 64);
    const uint64_t absorbed = r.u64(), perms = r.u64(), step_idx = r.u64(), has_prev = r.u64(),
                   val_obl = r.u64(), n_acc = r.u64();
    if (!r.ok || n_acc > sh->k_rho || has_prev > 1 || step_idx > 0xFFFFFFFFull)
        return ctx->fail(NEO_ERR_ARG, "shard_restore: malformed checkpoint");
    std::vector<MeInst> acc(n_acc);
    for (MeInst& me : acc) {
        r.vec(me.c);
        r.vec(me.X);
        r.vec(me.r);
        r.vec(me.y);
        r.vec(me.ysc);
        me.m_in = (uint32_t)r.u64();
        r.get(me.digest, 32);
        if (r.ok && (me.c.size() != (size_t)sh->kappa * NEO_D || me.r.size() != sh->ell_n))
            return ctx->fail(NEO_ERR_ARG, "shard_restore: malformed accumulator instance");
    }
    std::vector<uint64_t> prev_c, prev_X;
    r.vec(prev_c);
    r.vec(prev_X);
    std::vector<TwistInst> inits(sh->twist.size());
    for (auto& ti : inits) {
        r.vec(ti.init_addr);
        r.vec(ti.init_val);
        r.get(ti.digest, 32);
        if (r.ok && ti.init_addr.size() != ti.init_val.size())
            return ctx->fail(NEO_ERR_ARG, "shard_restore: malformed Twist init");
    }
    const uint64_t plane = (uint64_t)NEO_D * sh->m;
    uint64_t zb, vb, pb;
    const uint8_t* zsrc = r.blob(&zb);
    const uint8_t* vsrc = r.blob(&vb);
    const uint8_t* psrc = r.blob(&pb);
    if (!r.ok || r.left || zb != n_acc * plane || vb != (has_prev ? sh->valwit.bytes() : 0) ||
        pb != (has_prev ? sh->d_prev_cols.bytes() : 0))
        return ctx->fail(NEO_ERR_ARG, "shard_restore: malformed checkpoint");
    // everything validated: install
    NEO_CK(ctx, ctx_sync(ctx));
    if (zb) NEO_CK(ctx, cudaMemcpyAsync(sh->Zall.p + plane, zsrc, zb, cudaMemcpyHostToDevice, ctx->stream));
    if (vb) NEO_CK(ctx, cudaMemcpyAsync(sh->valwit.p, vsrc, vb, cudaMemcpyHostToDevice, ctx->stream));
    if (pb) NEO_CK(ctx, cudaMemcpyAsync(sh->d_prev_cols.p, psrc, pb, cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, ctx_sync(ctx));
    if (!sh->tr->restore(st, (uint32_t)absorbed, perms)) return ctx->fail(NEO_ERR_ARG, "shard_restore: bad transcript");
    sh->step_idx = (uint32_t)step_idx;
    sh->has_prev = has_prev != 0;
    sh->val_obligations = val_obl;
    sh->acc.swap(acc);
    sh->prev_c.swap(prev_c);
    sh->prev_X.swap(prev_X);
    for (size_t i = 0; i < inits.size(); i++) {
        sh->twist[i]->init_addr.swap(inits[i].init_addr);
        sh->twist[i]->init_val.swap(inits[i].init_val);
        memcpy(sh->twist[i]->digest, inits[i].digest, 32);
        sh->twist[i]->state_valid = false;
    }
    return NEO_OK;
}
extern "C" int neo_gpu_shard_restore(neo_gpu_shard* sh, const uint8_t* buf, uint64_t len) { NEO_ABI_GUARD(neo_gpu_shard_restore_impl_abi(sh, buf, len)) }
