// pp_gen.cu -- Ajtai public parameters generated on the device.
//
// The reference samples every PP coefficient by rejection from a ChaCha8
// stream: draw next_u64(), keep it if it is < q (sample_uniform_fq,
// crates/neo-ajtai/src/commit.rs:21-30).  `setup` (commit.rs:133-157) draws
// the whole kappa x m x 54 array from one stream; `setup_par`
// (commit.rs:159-225, and the seeded PP of commit.rs:227-264 used by
// shard.rs:776-800) draws kappa row seeds from the caller's stream, then per
// row one 32-byte seed per chunk of min(m, 2^15).max(1024) ring elements, and
// fills each chunk from its own ChaCha8 stream.
//
// ChaCha8 is counter based, so word w of a stream is block w/8 of the key
// stream: every thread computes one 64-byte block independently.  A word is
// rejected with probability (2^64 - q)/2^64 = 2^-32 - 2^-64, so a PP of
// 2^30 coefficients sees about one rejection in four generations.  The
// sampler therefore writes word w to output slot w (exact when nothing before
// it was rejected) and records every rejected position; only a stream that
// had a rejection is repaired, by a second pass that moves each accepted word
// w >= the first rejection to slot w - #(rejections before w).  Each stream is
// scanned `slack` words past its length so that the repair has the words it
// needs; if a stream has more rejections than slack the scan is redone with a
// larger slack.
#include "internal.cuh"
#include "transcript.h"

#include <algorithm>
#include <array>
#include <vector>

namespace {

constexpr uint32_t CC_THREADS = 256;
constexpr uint32_t CC_WORDS = 8;                         // u64 words per 64-byte ChaCha block
constexpr uint64_t CC_CTA_WORDS = (uint64_t)CC_THREADS * CC_WORDS;
constexpr uint32_t CC_PAD = CC_WORDS + 1;                // staging row stride (u64), breaks bank conflicts

__device__ __forceinline__ uint32_t rotl32(uint32_t x, int n) { return __funnelshift_l(x, x, n); }

// RFC 7539 block function with 8 rounds (4 double rounds), 64-bit block
// counter in words 12-13 and a zero nonce (rand_chacha ChaCha8Rng).
__device__ __forceinline__ void chacha8_block(const uint32_t (&key)[8], uint64_t ctr, uint32_t (&o)[16]) {
    uint32_t x[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                      key[4],      key[5],      key[6],      key[7],      (uint32_t)ctr, (uint32_t)(ctr >> 32),
                      0u,          0u};
#define NEO_CC_QR(a, b, c, d)                \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16); \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12); \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);  \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
#pragma unroll
    for (int r = 0; r < 4; r++) {
        NEO_CC_QR(0, 4, 8, 12) NEO_CC_QR(1, 5, 9, 13) NEO_CC_QR(2, 6, 10, 14) NEO_CC_QR(3, 7, 11, 15)
        NEO_CC_QR(0, 5, 10, 15) NEO_CC_QR(1, 6, 11, 12) NEO_CC_QR(2, 7, 8, 13) NEO_CC_QR(3, 4, 9, 14)
    }
#undef NEO_CC_QR
    const uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                            key[4],      key[5],      key[6],      key[7],      (uint32_t)ctr, (uint32_t)(ctr >> 32),
                            0u,          0u};
#pragma unroll
    for (int i = 0; i < 16; i++) o[i] = x[i] + s[i];
}

// Pass 1.  grid (CTAs over the longest stream, n_streams); CTA (x, s) covers
// words [x*2048, x*2048 + 2048) of stream s.  Words < count go to out[off + w]
// (staged through shared memory so each warp stores 256 contiguous bytes);
// words < count + slack that are >= bound are recorded in (rej_s, rej_w).
__global__ void __launch_bounds__(CC_THREADS) cc_sample_kernel(const uint32_t* __restrict__ keys,
                                                               const uint64_t* __restrict__ counts,
                                                               const uint64_t* __restrict__ offs, uint64_t slack,
                                                               uint64_t bound, uint64_t* __restrict__ out,
                                                               unsigned int* __restrict__ rej_n,
                                                               uint32_t* __restrict__ rej_s,
                                                               uint64_t* __restrict__ rej_w, uint32_t cap) {
    const uint32_t s = blockIdx.y;
    const uint64_t count = counts[s], limit = count + slack;
    const uint64_t cta_w0 = (uint64_t)blockIdx.x * CC_CTA_WORDS;
    if (cta_w0 >= limit) return;  // uniform over the CTA
    __shared__ uint64_t stage[CC_THREADS * CC_PAD];
    uint32_t key[8];
#pragma unroll
    for (int i = 0; i < 8; i++) key[i] = keys[s * 8 + i];
    const uint64_t blk = cta_w0 / CC_WORDS + threadIdx.x;
    uint32_t o[16];
    chacha8_block(key, blk, o);
#pragma unroll
    for (int k = 0; k < (int)CC_WORDS; k++) {
        const uint64_t v = (uint64_t)o[2 * k] | ((uint64_t)o[2 * k + 1] << 32);
        const uint64_t w = blk * CC_WORDS + k;
        if (v >= bound && w < limit) {
            const unsigned int idx = atomicAdd(rej_n, 1u);
            if (idx < cap) {
                rej_s[idx] = s;
                rej_w[idx] = w;
            }
        }
        stage[threadIdx.x * CC_PAD + k] = v;
    }
    __syncthreads();
    uint64_t* dst = out + offs[s];
#pragma unroll
    for (int i = 0; i < (int)CC_WORDS; i++) {
        const uint32_t j = threadIdx.x + i * CC_THREADS;  // word of the CTA's range
        const uint64_t w = cta_w0 + j;
        if (w < count) dst[w] = stage[(j / CC_WORDS) * CC_PAD + (j % CC_WORDS)];
    }
}

// Pass 2, for one stream with n_rej >= 1 rejections at sorted positions rej[]
// (all < limit, n_rej <= limit - count): accepted word w >= rej[0] goes to
// slot w - #(rej < w) when that slot is < count.  Slots below rej[0] keep what
// pass 1 wrote; every slot in [rej[0], count) is written exactly once.
__global__ void __launch_bounds__(CC_THREADS) cc_repair_kernel(const uint32_t* __restrict__ key8, uint64_t count,
                                                               uint64_t limit, uint64_t blk0,
                                                               const uint64_t* __restrict__ rej, uint32_t n_rej,
                                                               uint64_t bound, uint64_t* __restrict__ dst) {
    const uint64_t blk = blk0 + (uint64_t)blockIdx.x * CC_THREADS + threadIdx.x;
    if (blk * CC_WORDS >= limit) return;
    uint32_t key[8];
#pragma unroll
    for (int i = 0; i < 8; i++) key[i] = key8[i];
    uint32_t o[16];
    chacha8_block(key, blk, o);
    const uint64_t first = rej[0];
#pragma unroll
    for (int k = 0; k < (int)CC_WORDS; k++) {
        const uint64_t v = (uint64_t)o[2 * k] | ((uint64_t)o[2 * k + 1] << 32);
        const uint64_t w = blk * CC_WORDS + k;
        if (w >= limit || w < first || v >= bound) continue;
        uint32_t lo = 0, hi = n_rej;  // #(rej < w)
        while (lo < hi) {
            const uint32_t mid = (lo + hi) / 2;
            if (rej[mid] < w) lo = mid + 1;
            else hi = mid;
        }
        const uint64_t slot = w - lo;
        if (slot < count) dst[slot] = v;
    }
}

void key_words(const uint8_t* seed, uint32_t* key) {
    for (int i = 0; i < 8; i++)
        key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                 ((uint32_t)seed[4 * i + 3] << 24);
}

}  // namespace

// For each stream s (32-byte ChaCha8 seed seeds[s]), the first counts[s]
// words < bound of its next_u64() sequence, into d_out[offs[s] ...].
int chacha8_sample_device(neo_gpu_ctx* ctx, const uint8_t* seeds, uint32_t n_streams, const uint64_t* counts,
                          const uint64_t* offs, uint64_t bound, uint64_t* d_out) {
    if (n_streams == 0) return NEO_OK;
    if (n_streams > 65535) return ctx->fail(NEO_ERR_ARG, "chacha8_sample: at most 65535 streams");
    if (bound == 0) return ctx->fail(NEO_ERR_ARG, "chacha8_sample: bound must be > 0");
    std::vector<uint32_t> keys((size_t)n_streams * 8);
    uint64_t max_count = 0;
    double expected = 0;  // rejections per stream at the largest count
    for (uint32_t s = 0; s < n_streams; s++) {
        key_words(seeds + 32 * (size_t)s, &keys[8 * (size_t)s]);
        max_count = std::max(max_count, counts[s]);
    }
    if (max_count == 0) return NEO_OK;
    if (max_count > (1ull << 60)) return ctx->fail(NEO_ERR_ARG, "chacha8_sample: stream too long");
    expected = (double)max_count * ((double)(~bound) + 1.0) / 18446744073709551616.0;
    uint64_t slack = (uint64_t)(2.0 * expected) + 64;
    slack = (slack + CC_WORDS - 1) / CC_WORDS * CC_WORDS;

    DevBuf<uint32_t> d_keys;
    DevBuf<uint64_t> d_counts, d_offs;
    DevBuf<unsigned int> d_rej_n;
    NEO_CK(ctx, d_keys.alloc(keys.size()));
    NEO_CK(ctx, d_counts.alloc(n_streams));
    NEO_CK(ctx, d_offs.alloc(n_streams));
    NEO_CK(ctx, d_rej_n.alloc(1));
    NEO_CK(ctx, cudaMemcpyAsync(d_keys.p, keys.data(), d_keys.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(d_counts.p, counts, d_counts.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(d_offs.p, offs, d_offs.bytes(), cudaMemcpyHostToDevice, ctx->stream));

    std::vector<std::vector<uint64_t>> rej(n_streams);
    for (int attempt = 0;; attempt++) {
        if (attempt > 8) return ctx->fail(NEO_ERR_INVARIANT, "chacha8_sample: rejection slack did not converge");
        const uint64_t cap64 = std::max<uint64_t>(4096, (uint64_t)n_streams * slack);
        if (cap64 > (1u << 26)) return ctx->fail(NEO_ERR_ARG, "chacha8_sample: bound rejects too many words");
        const uint32_t cap = (uint32_t)cap64;
        DevBuf<uint32_t> d_rs;
        DevBuf<uint64_t> d_rw;
        NEO_CK(ctx, d_rs.alloc(cap));
        NEO_CK(ctx, d_rw.alloc(cap));
        NEO_CK(ctx, cudaMemsetAsync(d_rej_n.p, 0, sizeof(unsigned int), ctx->stream));
        const uint64_t ctas = (max_count + slack + CC_CTA_WORDS - 1) / CC_CTA_WORDS;
        if (ctas > 0x7fffffffull) return ctx->fail(NEO_ERR_ARG, "chacha8_sample: stream too long");
        cc_sample_kernel<<<dim3((uint32_t)ctas, n_streams), CC_THREADS, 0, ctx->stream>>>(
            d_keys.p, d_counts.p, d_offs.p, slack, bound, d_out, d_rej_n.p, d_rs.p, d_rw.p, cap);
        NEO_LAUNCHED(ctx);
        unsigned int n_rej = 0;
        NEO_CK(ctx, ctx_d2h(ctx, &n_rej, d_rej_n.p, sizeof n_rej));
        NEO_CK(ctx, ctx_sync(ctx));
        if (n_rej > cap) {
            // more rejections than the list holds: widen the slack so the list grows with it
            slack = std::max<uint64_t>(slack * 2, ((uint64_t)n_rej / n_streams + 1) * 2);
            slack = (slack + CC_WORDS - 1) / CC_WORDS * CC_WORDS;
            continue;
        }
        for (auto& r : rej) r.clear();
        if (n_rej) {
            std::vector<uint32_t> rs(n_rej);
            std::vector<uint64_t> rw(n_rej);
            NEO_CK(ctx, ctx_d2h(ctx, rs.data(), d_rs.p, (size_t)n_rej * 4));
            NEO_CK(ctx, ctx_d2h(ctx, rw.data(), d_rw.p, (size_t)n_rej * 8));
            NEO_CK(ctx, ctx_sync(ctx));
            for (uint32_t i = 0; i < n_rej; i++) rej[rs[i]].push_back(rw[i]);
        }
        uint64_t worst = 0;
        for (auto& r : rej) worst = std::max<uint64_t>(worst, r.size());
        if (worst <= slack) break;
        slack = (2 * worst + 64 + CC_WORDS - 1) / CC_WORDS * CC_WORDS;
    }
    for (uint32_t s = 0; s < n_streams; s++) {
        auto& r = rej[s];
        if (r.empty()) continue;
        std::sort(r.begin(), r.end());
        const uint64_t limit = counts[s] + slack;
        if (r[0] >= counts[s]) continue;  // rejections only past the stream's end: nothing moves
        DevBuf<uint64_t> d_r;
        NEO_CK(ctx, d_r.alloc(r.size()));
        NEO_CK(ctx, cudaMemcpyAsync(d_r.p, r.data(), d_r.bytes(), cudaMemcpyHostToDevice, ctx->stream));
        const uint64_t blk0 = r[0] / CC_WORDS, blk_end = (limit + CC_WORDS - 1) / CC_WORDS;
        const uint64_t ctas = (blk_end - blk0 + CC_THREADS - 1) / CC_THREADS;
        cc_repair_kernel<<<(uint32_t)ctas, CC_THREADS, 0, ctx->stream>>>(d_keys.p + 8 * (size_t)s, counts[s], limit,
                                                                         blk0, d_r.p, (uint32_t)r.size(), bound,
                                                                         d_out + offs[s]);
        NEO_LAUNCHED(ctx);
        NEO_CK(ctx, ctx_sync(ctx));  // d_r is freed on scope exit
    }
    return NEO_OK;
}

static int neo_gpu_chacha8_sample_impl_abi(neo_gpu_ctx* ctx, const uint8_t* seeds, uint32_t n_streams,
                                      const uint64_t* counts, uint64_t bound, uint64_t* out) {
    if (!ctx) return NEO_ERR_ARG;
    if ((n_streams && (!seeds || !counts)) || !out) return ctx->fail(NEO_ERR_ARG, "chacha8_sample: bad args");
    cudaSetDevice(ctx->device);
    std::vector<uint64_t> offs(n_streams);
    uint64_t total = 0;
    for (uint32_t s = 0; s < n_streams; s++) {
        offs[s] = total;
        total += counts[s];
    }
    if (total == 0) return NEO_OK;
    DevBuf<uint64_t> d_out;
    NEO_CK(ctx, d_out.alloc(total));
    int rc = chacha8_sample_device(ctx, seeds, n_streams, counts, offs.data(), bound, d_out.p);
    if (rc) return rc;
    NEO_CK(ctx, ctx_d2h(ctx, out, d_out.p, d_out.bytes()));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_chacha8_sample(neo_gpu_ctx* ctx, const uint8_t* seeds, uint32_t n_streams,
                                      const uint64_t* counts, uint64_t bound, uint64_t* out) { NEO_ABI_GUARD(neo_gpu_chacha8_sample_impl_abi(ctx, seeds, n_streams, counts, bound, out)) }

static int neo_gpu_pp_generate_impl_abi(neo_gpu_ctx* ctx, const uint8_t* seed, uint32_t kappa, uint64_t m, int mode) {
    if (!ctx) return NEO_ERR_ARG;
    if (!seed || kappa == 0 || kappa > 64 || m == 0) return ctx->fail(NEO_ERR_ARG, "pp_generate: bad args");
    if (mode != NEO_PP_SETUP && mode != NEO_PP_SETUP_PAR) return ctx->fail(NEO_ERR_ARG, "pp_generate: bad mode");
    cudaSetDevice(ctx->device);
    std::vector<std::array<uint8_t, 32>> seeds;
    std::vector<uint64_t> counts, offs;
    if (mode == NEO_PP_SETUP) {
        std::array<uint8_t, 32> s;
        std::copy(seed, seed + 32, s.begin());
        seeds.push_back(s);
        counts.push_back((uint64_t)kappa * m * NEO_D);
        offs.push_back(0);
    } else {
        // setup_par / seeded_pp_chunk_seeds: row seeds, then chunk seeds per row
        const uint64_t chunk = std::max<uint64_t>(std::min<uint64_t>(m, 1ull << 15), 1024);
        const uint64_t n_chunks = (m + chunk - 1) / chunk;
        neo::ChaCha8 master(seed);
        std::vector<std::array<uint8_t, 32>> rows(kappa);
        for (auto& r : rows) master.fill_bytes(r.data(), 32);
        for (uint32_t i = 0; i < kappa; i++) {
            neo::ChaCha8 rr(rows[i].data());
            for (uint64_t c = 0; c < n_chunks; c++) {
                std::array<uint8_t, 32> cs;
                rr.fill_bytes(cs.data(), 32);
                seeds.push_back(cs);
                const uint64_t lo = c * chunk, hi = std::min<uint64_t>(m, lo + chunk);
                counts.push_back((hi - lo) * NEO_D);
                offs.push_back(((uint64_t)i * m + lo) * NEO_D);
            }
        }
    }
    NEO_CK(ctx, ctx_sync(ctx));
    std::lock_guard<std::mutex> lk(pp_mutex());
    PPEntry* pp = nullptr;
    int rc = pp_slot(ctx, kappa, m, &pp);
    if (rc) return rc;
    pp->kappa = 0;  // not usable until the new coefficients are in place
    rc = chacha8_sample_device(ctx, seeds[0].data(), (uint32_t)seeds.size(), counts.data(), offs.data(), GL_Q,
                               pp->d_pp);
    if (rc) return rc;
    return pp_finish(ctx, pp, kappa);
}
extern "C" int neo_gpu_pp_generate(neo_gpu_ctx* ctx, const uint8_t* seed, uint32_t kappa, uint64_t m, int mode) { NEO_ABI_GUARD(neo_gpu_pp_generate_impl_abi(ctx, seed, kappa, m, mode)) }
