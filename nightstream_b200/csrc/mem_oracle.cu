// mem_oracle.cu -- Twist / Shout time-lane sum-check oracles on dense tables.
//
// Every time-lane oracle of crates/neo-memory/src/twist_oracle.rs is a sum over
// the time hypercube of a product of multilinear factors (bitness: χ times a
// weighted sum of b(b-1)).  The reference walks sparse columns pair by pair and
// recomputes χ_{r_cycle} children, eq-bit factors and, for Twist, Val_pre by a
// quadratic sum over all increments at every pair of every round
// (twist_oracle.rs:163-185, 311-379, 684-749).  Here each factor is a dense
// K table in HBM, built once:
//   * χ_{r_cycle} as a table, folded like any factor: folding variable 0 at c
//     multiplies by eq(c, r_0), which is the reference's prefix_eq update;
//   * eq_bit_affine(bit(t), r_b) per address bit: affine in the column, so
//     folding the factor equals the factor of the folded column;
//   * Val_pre(t) = init + Σ_{u<t} inc_terms(u): LT(u, ·) is the multilinear
//     extension of [u < t], so the reference's Σ inc_u·LT(u, point) is the
//     folded exclusive prefix sum (one scan here);
//   * LT(t, r_time) for the val-evaluation oracle.
// A round evaluates Σ_pairs Π_f (f0 + x (f1 - f0)) at x = 0..deg (one thread
// per (pair, x)), sums per block and then over blocks, and interpolates the
// requested points on the host. fold(r) is one pass over every factor.
// All arithmetic is exact in F_q / K, so values equal the reference's.
#include "internal.cuh"
#include <algorithm>

using gl::K;

namespace {

constexpr int MEM_MAX_DEG = 31;
constexpr int MT = 256;

__device__ __forceinline__ K shfl_xor_km(K a, int o) {
    K r;
    r.re = __shfl_xor_sync(0xffffffffu, a.re, o);
    r.im = __shfl_xor_sync(0xffffffffu, a.im, o);
    return r;
}

// eq(bit, u) = bit·(2u − 1) + (1 − u)   (neo-memory/src/bit_ops.rs:5-9)
__device__ __forceinline__ K eq_bit_affine(K bit, K u) {
    return gl::kadd(gl::kmul(bit, gl::ksub(gl::kdbl(u), gl::kone())), gl::ksub(gl::kone(), u));
}

// columns b < A of [A][len], in place: col_b[t] = eq_bit_affine(col_b[t], u_b)
__global__ void eqbit_kernel(K* __restrict__ cols, uint64_t len, uint32_t A, const K* __restrict__ u) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < len * A) cols[i] = eq_bit_affine(cols[i], u[i / len]);
}

// inc_terms(t) = has_write(t)·inc(t)·Π_b eq_bit_affine(wa_b(t), r_addr_b)
// (build_inc_terms_at_r_addr, twist_oracle.rs:351-378)
__global__ void inc_terms_kernel(const K* __restrict__ has_w, const K* __restrict__ inc, const K* __restrict__ wa,
                                 uint32_t A, const K* __restrict__ r_addr, uint64_t len, K* __restrict__ out) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= len) return;
    K v = gl::kmul(has_w[t], inc[t]);
    for (uint32_t b = 0; b < A; b++) v = gl::kmul(v, eq_bit_affine(wa[(uint64_t)b * len + t], r_addr[b]));
    out[t] = v;
}

// exclusive prefix sum over K in three passes: per-block sums, a scan of the
// block sums (one block), and the per-element scan with the block offset.
constexpr int SCAN_T = 256, SCAN_E = 4, SCAN_BLK = SCAN_T * SCAN_E;

__device__ K block_excl_scan(K v, K* s_warp, K* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    K inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        K n;
        n.re = __shfl_up_sync(0xffffffffu, inc.re, o);
        n.im = __shfl_up_sync(0xffffffffu, inc.im, o);
        if (lane >= o) inc = gl::kadd(inc, n);
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        K w = lane < nw ? s_warp[lane] : gl::kzero();
        K wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            K n;
            n.re = __shfl_up_sync(0xffffffffu, wi.re, o);
            n.im = __shfl_up_sync(0xffffffffu, wi.im, o);
            if (lane >= o) wi = gl::kadd(wi, n);
        }
        if (lane < nw) s_warp[lane] = gl::ksub(wi, w);  // exclusive warp offsets
        if (lane == nw - 1) *total = wi;
    }
    __syncthreads();
    K r = gl::kadd(s_warp[warp], gl::ksub(inc, v));
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_T) scan_sums_kernel(const K* __restrict__ in, uint64_t len, K* __restrict__ sums) {
    __shared__ K s_warp[32];
    __shared__ K s_tot;
    uint64_t base = blockIdx.x * (uint64_t)SCAN_BLK + threadIdx.x * SCAN_E;
    K v = gl::kzero();
#pragma unroll
    for (int e = 0; e < SCAN_E; e++)
        if (base + e < len) v = gl::kadd(v, in[base + e]);
    block_excl_scan(v, s_warp, &s_tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = s_tot;
}

// one block scans up to SCAN_T * chunk block sums, in place, exclusive, plus init
__global__ void __launch_bounds__(SCAN_T) scan_top_kernel(K* __restrict__ sums, uint32_t n, K init) {
    __shared__ K s_warp[32];
    __shared__ K s_tot;
    K carry = init;
    for (uint32_t base = 0; base < n; base += SCAN_T) {
        uint32_t i = base + threadIdx.x;
        K v = i < n ? sums[i] : gl::kzero();
        K ex = block_excl_scan(v, s_warp, &s_tot);
        if (i < n) sums[i] = gl::kadd(carry, ex);
        carry = gl::kadd(carry, s_tot);
        __syncthreads();
    }
}

// out = prefix(in) combined per kind:
//   combine 0: out = VP                      (plain exclusive prefix + init)
//   combine 1: out = VP − a                  (read check:  Val_pre − rv)
//   combine 2: out = a − VP − b              (write check: wv − Val_pre − inc)
__global__ void __launch_bounds__(SCAN_T) scan_final_kernel(const K* __restrict__ in, uint64_t len,
                                                            const K* __restrict__ offs, int combine,
                                                            const K* __restrict__ a, const K* __restrict__ b,
                                                            K* __restrict__ out) {
    __shared__ K s_warp[32];
    __shared__ K s_tot;
    uint64_t base = blockIdx.x * (uint64_t)SCAN_BLK + threadIdx.x * SCAN_E;
    K v[SCAN_E];
    K s = gl::kzero();
#pragma unroll
    for (int e = 0; e < SCAN_E; e++) {
        v[e] = base + e < len ? in[base + e] : gl::kzero();
        s = gl::kadd(s, v[e]);
    }
    K run = gl::kadd(offs[blockIdx.x], block_excl_scan(s, s_warp, &s_tot));
#pragma unroll
    for (int e = 0; e < SCAN_E; e++) {
        uint64_t t = base + e;
        if (t < len) {
            K o = run;
            if (combine == 1) o = gl::ksub(run, a[t]);
            else if (combine == 2) o = gl::ksub(gl::ksub(a[t], run), b[t]);
            out[t] = o;
        }
        run = gl::kadd(run, v[e]);
    }
}

// LT(t, r) for Boolean t (twist_oracle.rs:320-334)
__global__ void lt_table_kernel(const K* __restrict__ r, uint32_t ell, K* __restrict__ out) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= (1ULL << ell)) return;
    K suffix = gl::kone(), acc = gl::kzero();
    for (int i = (int)ell - 1; i >= 0; i--) {
        K ri = r[i];
        if (((t >> i) & 1) == 0) {
            acc = gl::kadd(acc, gl::kmul(ri, suffix));
            suffix = gl::kmul(suffix, gl::ksub(gl::kone(), ri));
        } else {
            suffix = gl::kmul(suffix, ri);
        }
    }
    out[t] = acc;
}

// fold every factor on variable 0: dst[f][p] = src[f][2p] + r (src[f][2p+1] − src[f][2p])
__global__ void mem_fold_kernel(const K* __restrict__ src, uint64_t src_len, K* __restrict__ dst, uint32_t nf, K r) {
    const uint64_t half = src_len >> 1;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= half * nf) return;
    uint64_t f = i / half, p = i - f * half;
    const K* s = src + f * src_len + 2 * p;
    dst[f * half + p] = gl::klerp(s[0], s[1], r);
}

struct MemEvalArgs {
    const K* tab;       // [nf][len]
    uint64_t len;       // current table length (>= 2)
    uint32_t nf;
    int bitness;        // 1: factor 0 is χ, the rest columns weighted by w
    const K* w;         // bitness weights [nf - 1]
    K* partials;        // [npts][gridDim.x]
};

// one thread per (pair, x); x = blockIdx.y
__global__ void __launch_bounds__(MT) mem_eval_kernel(const MemEvalArgs a) {
    __shared__ K s_red[MT / 32];
    const uint64_t pairs = a.len >> 1;
    const uint64_t p = blockIdx.x * (uint64_t)MT + threadIdx.x;
    const uint32_t x = blockIdx.y;
    K acc = gl::kzero();
    if (p < pairs) {
        // A factor that is zero on both children makes the whole product zero
        // at every x: gate columns (has_lookup, has_read, has_write, the
        // address weights) are zero outside the active trace rows, so most
        // pairs stop after loading the gate (factors are ordered gate-first).
        if (!a.bitness) {
            K prod = gl::kone();
            for (uint32_t f = 0; f < a.nf; f++) {
                const K* s = a.tab + (uint64_t)f * a.len + 2 * p;
                K f0 = s[0], f1 = s[1];
                if (gl::kiszero(f0) && gl::kiszero(f1)) {
                    prod = gl::kzero();
                    break;
                }
                K v = gl::kadd(f0, gl::kscale_small(gl::ksub(f1, f0), (int32_t)x));
                prod = gl::kmul(prod, v);
            }
            acc = prod;
        } else {
            const K* s = a.tab + 2 * p;
            K sum = gl::kzero();
            for (uint32_t f = 1; f < a.nf; f++) {
                const K* c = a.tab + (uint64_t)f * a.len + 2 * p;
                if (gl::kiszero(c[0]) && gl::kiszero(c[1])) continue;  // b(b - 1) = 0 at every x
                K bx = gl::kadd(c[0], gl::kscale_small(gl::ksub(c[1], c[0]), (int32_t)x));
                sum = gl::kadd(sum, gl::kmul(gl::kmul(a.w[f - 1], bx), gl::ksub(bx, gl::kone())));
            }
            if (!gl::kiszero(sum)) {
                K chi = gl::kadd(s[0], gl::kscale_small(gl::ksub(s[1], s[0]), (int32_t)x));
                acc = gl::kmul(chi, sum);
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = gl::kadd(acc, shfl_xor_km(acc, o));
    if (lane == 0) s_red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        K s = gl::kzero();
#pragma unroll
        for (int w = 0; w < MT / 32; w++) s = gl::kadd(s, s_red[w]);
        a.partials[(uint64_t)x * gridDim.x + blockIdx.x] = s;
    }
}

// vals[x] = Σ_b partials[x][b]; one block per x
__global__ void __launch_bounds__(256) mem_reduce_kernel(const K* __restrict__ partials, uint32_t nblocks,
                                                         K* __restrict__ vals) {
    __shared__ K s_red[8];
    const uint32_t x = blockIdx.x;
    K v = gl::kzero();
    for (uint32_t b = threadIdx.x; b < nblocks; b += blockDim.x) v = gl::kadd(v, partials[(uint64_t)x * nblocks + b]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_km(v, o));
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        K s = gl::kzero();
        for (int w = 0; w < 8; w++) s = gl::kadd(s, s_red[w]);
        vals[x] = s;
    }
}

// AddressLookupOracle weight table (twist_oracle.rs:1671-1724):
// w[addr(t)] += χ_{r_cycle}(t)·has_lookup(t), addr from bit columns equal to 1.
// Exact order-free accumulation: each u64 component is summed with a 64-bit
// atomic and its carries are counted separately (sum = lo + 2^64·carries).
__global__ void addr_weights_kernel(const K* __restrict__ chi, const K* __restrict__ has, const K* __restrict__ bits,
                                    uint32_t A, uint64_t len, unsigned long long* __restrict__ lo,
                                    unsigned long long* __restrict__ carry) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= len) return;
    K g = has[t];
    if (gl::kiszero(g)) return;
    K wt = gl::kmul(chi[t], g);
    if (gl::kiszero(wt)) return;
    uint64_t addr = 0;
    for (uint32_t b = 0; b < A; b++) {
        K v = bits[(uint64_t)b * len + t];
        if (v.re == 1 && v.im == 0) addr |= 1ULL << b;
    }
    unsigned long long o = atomicAdd(&lo[2 * addr], (unsigned long long)wt.re);
    if (o + wt.re < o) atomicAdd(&carry[2 * addr], 1ULL);
    o = atomicAdd(&lo[2 * addr + 1], (unsigned long long)wt.im);
    if (o + wt.im < o) atomicAdd(&carry[2 * addr + 1], 1ULL);
}

__global__ void addr_weights_finish_kernel(const unsigned long long* __restrict__ lo,
                                           const unsigned long long* __restrict__ carry, uint64_t n, K* __restrict__ w) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    // lo + carry·2^64 with 2^64 = 2^32 − 1 (mod q)
    uint64_t re = gl::add(gl::canon(lo[2 * i]), gl::mul(gl::canon(carry[2 * i]), GL_EPS));
    uint64_t im = gl::add(gl::canon(lo[2 * i + 1]), gl::mul(gl::canon(carry[2 * i + 1]), GL_EPS));
    w[i] = gl::kmk(re, im);
}

// claim = Σ_a table[a]·w[a] (block partials, reduced by mem_reduce_kernel)
__global__ void __launch_bounds__(256) dot_kernel(const K* __restrict__ a, const K* __restrict__ b, uint64_t n,
                                                  K* __restrict__ partials) {
    __shared__ K s_red[8];
    K v = gl::kzero();
    for (uint64_t i = blockIdx.x * 256ULL + threadIdx.x; i < n; i += 256ULL * gridDim.x)
        v = gl::kadd(v, gl::kmul(a[i], b[i]));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_km(v, o));
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        K s = gl::kzero();
        for (int w = 0; w < 8; w++) s = gl::kadd(s, s_red[w]);
        partials[blockIdx.x] = s;
    }
}

// ---- all memory claims of one sum-check round in one launch --------------
// A batched round (the Route-A time claims, the val-eval batch, the address
// pre-time batches) evaluates every claim's round polynomial at x = 0..deg
// before the transcript draws the next challenge.  One kernel folds (the
// pending challenge), evaluates and reduces (each claim's last block sums its
// partials) the tables of up to MULTI_MAX claims together; the values land in
// one device array that the host reads with a single copy.
constexpr int MULTI_MAX = 24;
constexpr int MX = 8;  // evaluation points per pass (thread-local accumulators)

struct MultiClaim {
    const K* tab;      // [nf][len] current tables (written by this launch when src is set)
    const K* src;      // a pending fold: [nf][2 len] tables before binding r, else null
    uint64_t len;
    uint32_t nf, npts;
    int bitness;
    const K* w;        // bitness weights [nf - 1]
    K r;               // fold challenge
    uint32_t blk0;     // first block of this claim
    uint32_t part0;    // first partial [npts][nblk]
    uint32_t nblk;     // partial columns per point: pair blocks of 256 pairs x column chunks
    uint32_t ppt;      // evaluation points per thread (1, 2, 4 or MX): blocks = ceil(npts / ppt) * nblk
    uint32_t nchunk;   // bitness: column chunks of BIT_CHUNK columns (1 otherwise)
    K* out;            // values at x = 0..npts-1
    unsigned int* ticket;  // the claim's block counter (zero between launches)
};
constexpr uint32_t BIT_CHUNK = 4;  // bitness columns per thread

struct MultiArgs {
    int n;
    MultiClaim c[MULTI_MAX];
    K* partials;
};

__device__ __forceinline__ int multi_claim_of(const MultiArgs& a, uint32_t blk) {
    int c = 0;
    while (c + 1 < a.n && blk >= a.c[c + 1].blk0) c++;
    return c;
}

// Factor f of pair p in the current round: (f0, f1) = the entries 2p, 2p+1.
// With a pending fold they are lerp(src[4p], src[4p+1], r) and lerp(src[4p+2],
// src[4p+3], r) -- computed here unless this thread wrote them already.
__device__ __forceinline__ void multi_factor(const MultiClaim& c, uint32_t f, uint64_t p, bool from_tab, K& f0, K& f1) {
    if (c.src && !from_tab) {
        const K* o = c.src + (uint64_t)f * (2 * c.len) + 4 * p;
        f0 = gl::klerp(o[0], o[1], c.r);
        f1 = gl::klerp(o[2], o[3], c.r);
        return;
    }
    const K* s = c.tab + (uint64_t)f * c.len + 2 * p;
    f0 = s[0];
    f1 = s[1];
}

// The pending fold of the factors this thread owns (point group 0: every
// factor, or for a bitness claim its column chunk and, in chunk 0, chi).
__device__ __forceinline__ void multi_fold_owned(const MultiClaim& c, uint64_t p, uint32_t ch) {
    K* t = const_cast<K*>(c.tab);
    auto one = [&](uint32_t f) {
        const K* o = c.src + (uint64_t)f * (2 * c.len) + 4 * p;
        t[(uint64_t)f * c.len + 2 * p] = gl::klerp(o[0], o[1], c.r);
        t[(uint64_t)f * c.len + 2 * p + 1] = gl::klerp(o[2], o[3], c.r);
    };
    if (!c.bitness) {
        for (uint32_t f = 0; f < c.nf; f++) one(f);
        return;
    }
    if (ch == 0) one(0);
    const uint32_t f_lo = 1 + ch * BIT_CHUNK, f_hi = min(c.nf, f_lo + BIT_CHUNK);
    for (uint32_t f = f_lo; f < f_hi; f++) one(f);
}

// Values of one pair at x = x0 .. x0 + PPT - 1: the product of the claim's
// affine factors (a factor zero on both children zeroes every point), or for
// a bitness claim chi(x) times the weighted b(b - 1) sum over the columns of
// chunk ch, additions along x.  own: this thread folded its factors already.
template <int PPT>
__device__ __forceinline__ void multi_eval_points(const MultiClaim& c, uint64_t p, uint32_t x0, uint32_t ch, bool own,
                                                  K* acc) {
    if (!c.bitness) {
#pragma unroll
        for (int i = 0; i < PPT; i++) acc[i] = gl::kone();
        for (uint32_t f = 0; f < c.nf; f++) {
            K f0, f1;
            multi_factor(c, f, p, own, f0, f1);
            if (gl::kiszero(f0) && gl::kiszero(f1)) {
#pragma unroll
                for (int i = 0; i < PPT; i++) acc[i] = gl::kzero();
                return;
            }
            const K d = gl::ksub(f1, f0);
            K v = gl::kadd(f0, gl::kscale_small(d, (int32_t)x0));
#pragma unroll
            for (int i = 0; i < PPT; i++) {
                acc[i] = gl::kmul(acc[i], v);
                v = gl::kadd(v, d);
            }
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < PPT; i++) acc[i] = gl::kzero();
    const uint32_t f_lo = 1 + ch * BIT_CHUNK, f_hi = min(c.nf, f_lo + BIT_CHUNK);
    // the chunk's column pairs are loaded together (one memory round trip)
    K b0[BIT_CHUNK], b1[BIT_CHUNK];
#pragma unroll
    for (uint32_t u = 0; u < BIT_CHUNK; u++) {
        if (f_lo + u < f_hi) multi_factor(c, f_lo + u, p, own, b0[u], b1[u]);
        else b0[u] = b1[u] = gl::kzero();
    }
    bool any = false;
#pragma unroll
    for (uint32_t u = 0; u < BIT_CHUNK; u++) {
        if (gl::kiszero(b0[u]) && gl::kiszero(b1[u])) continue;  // b(b - 1) = 0 at every x
        any = true;
        const K d = gl::ksub(b1[u], b0[u]), w = c.w[f_lo + u - 1];
        K v = gl::kadd(b0[u], gl::kscale_small(d, (int32_t)x0));
#pragma unroll
        for (int i = 0; i < PPT; i++) {
            acc[i] = gl::kadd(acc[i], gl::kmul(w, gl::kmul(v, gl::ksub(v, gl::kone()))));
            v = gl::kadd(v, d);
        }
    }
    if (!any) return;
    K f0, f1;
    multi_factor(c, 0, p, own && ch == 0, f0, f1);
    const K d = gl::ksub(f1, f0);
    K v = gl::kadd(f0, gl::kscale_small(d, (int32_t)x0));
#pragma unroll
    for (int i = 0; i < PPT; i++) {
        acc[i] = gl::kmul(acc[i], v);
        v = gl::kadd(v, d);
    }
}

// Block (point group g, partial column r) of one claim: r = ch * (pair
// blocks) + pair block pb; thread t takes pair pb * 256 + t (bitness: its
// column chunk ch) at the claim's ppt points x0 = g * ppt ..; each point is
// reduced over the block into partials[x][r].  A claim with many pairs takes
// MX points per thread (its factor pairs read once per MX points); one with
// few pairs (the late rounds) takes fewer, so that its point groups run side
// by side instead of one thread walking every point.
__global__ void __launch_bounds__(256) mem_multi_eval_kernel(const __grid_constant__ MultiArgs a) {
    __shared__ K s_red[256 / 32][MX];
    const int ci = multi_claim_of(a, blockIdx.x);
    const MultiClaim& c = a.c[ci];
    const uint32_t b = blockIdx.x - c.blk0;
    const uint32_t g = b / c.nblk, pb = b % c.nblk;  // pb: the partial column
    const uint32_t nbp = c.nblk / c.nchunk;          // pair blocks
    const uint32_t ch = pb / nbp;
    const uint32_t x0 = g * c.ppt;
    const uint32_t np = min(c.ppt, c.npts - x0);
    const uint64_t pairs = c.len >> 1;
    const uint64_t p = (uint64_t)(pb % nbp) * 256 + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // a product whose gate factor (factor 1: has_lookup / has_read /
    // has_write behind chi; factor 0 where no chi leads) is zero on both
    // children contributes nothing at any x
    bool live = p < pairs;
    // a pending fold: point group 0 writes the folded tables of its pairs
    const bool own = c.src && g == 0;
    if (live && own) multi_fold_owned(c, p, ch);
    if (live && !c.bitness) {
        K a0, a1, b0, b1;
        multi_factor(c, 0, p, own, a0, a1);
        multi_factor(c, c.nf > 1 ? 1 : 0, p, own, b0, b1);
        live = !(gl::kiszero(a0) && gl::kiszero(a1)) && !(gl::kiszero(b0) && gl::kiszero(b1));
    }
    K acc[MX];
#pragma unroll
    for (int i = 0; i < MX; i++) acc[i] = gl::kzero();
    if (live) {
        switch (c.ppt) {
            case 1: multi_eval_points<1>(c, p, x0, ch, own, acc); break;
            case 2: multi_eval_points<2>(c, p, x0, ch, own, acc); break;
            case 4: multi_eval_points<4>(c, p, x0, ch, own, acc); break;
            default: multi_eval_points<MX>(c, p, x0, ch, own, acc); break;
        }
    }
    const bool any = __syncthreads_or(live);
    if (!any) {
        if (threadIdx.x < np) a.partials[c.part0 + (uint64_t)(x0 + threadIdx.x) * c.nblk + pb] = gl::kzero();
    } else {
#pragma unroll
        for (int i = 0; i < MX; i++) {
            if ((uint32_t)i >= np) break;
            K v = acc[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_km(v, o));
            if (lane == 0) s_red[warp][i] = v;
        }
        __syncthreads();
        if (threadIdx.x < np) {
            K v = gl::kzero();
#pragma unroll
            for (int w = 0; w < 256 / 32; w++) v = gl::kadd(v, s_red[w][threadIdx.x]);
            a.partials[c.part0 + (uint64_t)(x0 + threadIdx.x) * c.nblk + pb] = v;
        }
    }
    // the claim's last block to finish sums its partials (ticket, no waits)
    __threadfence();
    __syncthreads();
    __shared__ unsigned int s_last;
    const uint32_t claim_blocks = c.nblk * ((c.npts + c.ppt - 1) / c.ppt);
    if (threadIdx.x == 0) s_last = atomicInc(c.ticket, claim_blocks - 1) == claim_blocks - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // one warp per point: the points' sums run side by side (a claim of the
    // late rounds has one partial per point, so this tail is a few load
    // latencies instead of one block-wide reduction per point)
    for (uint32_t x = warp; x < c.npts; x += 256 / 32) {
        K v = gl::kzero();
#pragma unroll 4
        for (uint32_t r = lane; r < c.nblk; r += 32) {
            const ulonglong2 u = __ldcg(reinterpret_cast<const ulonglong2*>(a.partials + c.part0 + (uint64_t)x * c.nblk + r));
            v = gl::kadd(v, gl::kmk(u.x, u.y));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_km(v, o));
        if (lane == 0) c.out[x] = v;
    }
}


inline K kload_h(const uint64_t* p) { return gl::kmk(p[0], p[1]); }

}  // namespace

struct neo_gpu_mem_oracle {
    neo_gpu_ctx* ctx = nullptr;
    int kind = 0;
    uint32_t ell = 0, A = 0, deg = 0, nf = 0, bit_idx = 0;
    int bitness = 0;
    uint64_t len = 0;     // current table length
    DevBuf<K> tab[2];     // ping-pong factor tables [nf][len]
    int cur = 0;
    bool pending = false; // a fold challenge not yet applied
    K pending_r{};
    DevBuf<K> w;          // bitness weights
    std::vector<K> hw;    // host copy of the weights
    DevBuf<K> partials, vals;
    DevBuf<K> dpt, dra, tmp, sums;  // build workspace, kept for reuse
    std::vector<K> hvals;
    K claim{};
};

namespace {

uint32_t factor_count(int kind, uint32_t A, uint32_t n_cols) {
    switch (kind) {
        case NEO_MEM_SHOUT_VALUE: return 3;
        case NEO_MEM_SHOUT_ADAPTER: return 2 + A;
        case NEO_MEM_BITNESS: return 1 + n_cols;
        case NEO_MEM_TWIST_READ: return 3 + A;
        case NEO_MEM_TWIST_WRITE: return 3 + A;
        case NEO_MEM_VAL_EVAL: return 3 + A;
        case NEO_MEM_TOTAL_INC: return 2 + A;
        case NEO_MEM_PRODUCT: return n_cols;
    }
    return 0;
}

int expected_cols(int kind, uint32_t A, uint32_t n_cols) {
    switch (kind) {
        case NEO_MEM_SHOUT_VALUE: return 2;
        case NEO_MEM_SHOUT_ADAPTER: return 1 + A;
        case NEO_MEM_BITNESS: return n_cols;
        case NEO_MEM_TWIST_READ: return 4 + 2 * A;
        case NEO_MEM_TWIST_WRITE: return 3 + A;
        case NEO_MEM_VAL_EVAL: case NEO_MEM_TOTAL_INC: return 2 + A;
        case NEO_MEM_PRODUCT: return n_cols;
    }
    return -1;
}

uint32_t degree_of(int kind, uint32_t A, uint32_t n_cols) {
    switch (kind) {
        case NEO_MEM_SHOUT_VALUE: case NEO_MEM_BITNESS: return 3;
        case NEO_MEM_SHOUT_ADAPTER: case NEO_MEM_TOTAL_INC: return 2 + A;
        case NEO_MEM_TWIST_READ: case NEO_MEM_TWIST_WRITE: case NEO_MEM_VAL_EVAL: return 3 + A;
        case NEO_MEM_PRODUCT: return n_cols;
    }
    return 0;
}

// round values at x = 0..deg into o->hvals (applies a pending fold first)
int mem_round_values(neo_gpu_mem_oracle* o) {
    neo_gpu_ctx* ctx = o->ctx;
    if (o->pending) {
        K* src = o->tab[o->cur].p;
        K* dst = o->tab[o->cur ^ 1].p;
        uint64_t tot = (o->len >> 1) * o->nf;
        mem_fold_kernel<<<ceil_div(tot, 256), 256, 0, ctx->stream>>>(src, o->len, dst, o->nf, o->pending_r);
        NEO_LAUNCHED(ctx);
        o->cur ^= 1;
        o->len >>= 1;
        o->pending = false;
    }
    const uint32_t npts = o->deg + 1;
    o->hvals.assign(npts, gl::kzero());
    if (o->len == 1) {
        std::vector<K> v(o->nf);
        NEO_CK(ctx, ctx_d2h(ctx, v.data(), o->tab[o->cur].p, o->nf * sizeof(K)));
        NEO_CK(ctx, ctx_sync(ctx));
        K val;
        if (o->bitness) {
            K s = gl::kzero();
            for (uint32_t f = 1; f < o->nf; f++)
                s = gl::kadd(s, gl::kmul(gl::kmul(o->hw[f - 1], v[f]), gl::ksub(v[f], gl::kone())));
            val = gl::kmul(v[0], s);
        } else {
            val = gl::kone();
            for (uint32_t f = 0; f < o->nf; f++) val = gl::kmul(val, v[f]);
        }
        for (auto& h : o->hvals) h = val;
        return NEO_OK;
    }
    const uint64_t pairs = o->len >> 1;
    const uint32_t nb = (uint32_t)ceil_div(pairs, MT);
    NEO_CK(ctx, o->partials.ensure((size_t)nb * npts));
    MemEvalArgs a;
    a.tab = o->tab[o->cur].p;
    a.len = o->len;
    a.nf = o->nf;
    a.bitness = o->bitness;
    a.w = o->w.p;
    a.partials = o->partials.p;
    mem_eval_kernel<<<dim3(nb, npts), MT, 0, ctx->stream>>>(a);
    NEO_LAUNCHED(ctx);
    mem_reduce_kernel<<<npts, 256, 0, ctx->stream>>>(o->partials.p, nb, o->vals.p);
    NEO_LAUNCHED(ctx);
    NEO_CK(ctx, ctx_d2h(ctx, o->hvals.data(), o->vals.p, npts * sizeof(K)));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}

// p(x) from p(0..n-1) (Lagrange on the integer nodes)
K lagrange_at(const std::vector<K>& v, K x) {
    const int n = (int)v.size();
    if (x.im == 0 && x.re < (uint64_t)n) return v[x.re];
    K acc = gl::kzero();
    for (int i = 0; i < n; i++) {
        K num = gl::kone();
        uint64_t den = 1;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            num = gl::kmul(num, gl::ksub(x, gl::kfq((uint64_t)j)));
            den = gl::mul(den, i > j ? (uint64_t)(i - j) : gl::neg((uint64_t)(j - i)));
        }
        acc = gl::kadd(acc, gl::kmul(v[i], gl::kscale(num, gl::inv(den))));
    }
    return acc;
}

int mem_create(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point, uint32_t A, const uint64_t* r_addr,
               const uint64_t* init, uint32_t n_cols, const uint64_t* cols, bool cols_on_device,
               const uint64_t* weights, uint64_t* claim_out, neo_gpu_mem_oracle** out, bool reuse = false,
               bool lazy = false) {
    if (!ctx || !out) return NEO_ERR_ARG;
    if (!reuse) *out = nullptr;
    if (kind < NEO_MEM_SHOUT_VALUE || kind > NEO_MEM_PRODUCT) return ctx->fail(NEO_ERR_ARG, "mem_oracle: unknown kind");
    if (ell > 30) return ctx->fail(NEO_ERR_ARG, "mem_oracle: ell > 30");
    if (expected_cols(kind, A, n_cols) != (int)n_cols || (n_cols == 0 && kind != NEO_MEM_BITNESS))
        return ctx->fail(NEO_ERR_ARG, "mem_oracle: column count does not match the kind");
    const bool chi = kind <= NEO_MEM_TWIST_WRITE;
    if ((chi || kind == NEO_MEM_VAL_EVAL) && !r_point) return ctx->fail(NEO_ERR_ARG, "mem_oracle: missing r_cycle / r_time");
    if (A && !r_addr && kind != NEO_MEM_BITNESS && kind != NEO_MEM_PRODUCT && kind != NEO_MEM_SHOUT_VALUE)
        return ctx->fail(NEO_ERR_ARG, "mem_oracle: missing r_addr");
    if (kind == NEO_MEM_BITNESS && !weights && n_cols) return ctx->fail(NEO_ERR_ARG, "mem_oracle: missing weights");
    if (!cols && n_cols) return ctx->fail(NEO_ERR_ARG, "mem_oracle: null columns");
    const uint32_t deg = degree_of(kind, A, n_cols);
    if (deg > MEM_MAX_DEG) return ctx->fail(NEO_ERR_UNSUPPORTED, "mem_oracle: degree bound above 31");
    cudaSetDevice(ctx->device);

    // reuse: rebuild into the caller's object, keeping its device buffers
    neo_gpu_mem_oracle* o = reuse ? *out : nullptr;
    const bool fresh = !o;
    if (fresh) o = new neo_gpu_mem_oracle();
    o->ctx = ctx;
    o->bit_idx = 0;
    o->cur = 0;
    o->pending = false;
    o->hw.clear();
    o->kind = kind;
    o->ell = ell;
    o->A = A;
    o->deg = deg;
    o->nf = factor_count(kind, A, n_cols);
    o->bitness = kind == NEO_MEM_BITNESS;
    o->len = 1ULL << ell;
    const uint64_t L = o->len;
    auto fail = [&](int rc) {
        if (fresh) delete o;
        return rc;
    };
    if (o->tab[0].ensure((size_t)o->nf * L) || o->tab[1].ensure((size_t)o->nf * (L > 1 ? L / 2 : 1)) ||
        o->vals.ensure(deg + 1))
        return fail(ctx->fail(NEO_ERR_OOM, "mem_oracle: table allocation"));
    K* T = o->tab[0].p;
    cudaStream_t S = ctx->stream;
    const cudaMemcpyKind cpk = cols_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const size_t colb = L * sizeof(K);
    auto col = [&](uint32_t c) { return reinterpret_cast<const K*>(cols) + (size_t)c * L; };
    auto put = [&](uint32_t f, uint32_t c) { return cudaMemcpyAsync(T + (size_t)f * L, col(c), colb, cpk, S); };
    DevBuf<K>& dpt = o->dpt;
    DevBuf<K>& dra = o->dra;
    DevBuf<K>& tmp = o->tmp;
    if (r_point && dpt.ensure(ell ? ell : 1)) return fail(ctx->fail(NEO_ERR_OOM, "mem_oracle: point"));
    if (r_point && ell && cudaMemcpyAsync(dpt.p, r_point, ell * sizeof(K), cudaMemcpyHostToDevice, S))
        return fail(ctx->fail(NEO_ERR_CUDA, "mem_oracle: point upload"));
    if (A && r_addr) {
        if (dra.ensure(A) || cudaMemcpyAsync(dra.p, r_addr, A * sizeof(K), cudaMemcpyHostToDevice, S))
            return fail(ctx->fail(NEO_ERR_OOM, "mem_oracle: r_addr"));
    }
    auto eqbits = [&](uint32_t f0, uint32_t c0) -> int {
        if (!A) return NEO_OK;
        if (!r_addr) return ctx->fail(NEO_ERR_ARG, "mem_oracle: address bits without r_addr");
        for (uint32_t b = 0; b < A; b++)
            if (put(f0 + b, c0 + b)) return ctx->fail(NEO_ERR_CUDA, "mem_oracle: column upload");
        eqbit_kernel<<<ceil_div(L * A, 256), 256, 0, S>>>(T + (size_t)f0 * L, L, A, dra.p);  // all A columns at once
        NEO_LAUNCHED(ctx);
        return NEO_OK;
    };
    int rc = NEO_OK;
    if (chi) {  // factor 0 = χ_{r_cycle}, copied when the previous oracle built it for the same point
        std::vector<uint64_t> key(1, ell);
        key.insert(key.end(), r_point, r_point + 2 * (size_t)ell);
        const size_t bytes = L * sizeof(K);
        if (ctx->chi_cache && ctx->chi_key == key && ctx->chi_cache_bytes >= bytes) {
            if (cudaMemcpyAsync(T, ctx->chi_cache, bytes, cudaMemcpyDeviceToDevice, S))
                return fail(ctx->fail(NEO_ERR_CUDA, "mem_oracle: chi copy"));
        } else {
            rc = launch_chi_table(ctx, dpt.p, ell, T);
            if (rc) return fail(rc);
            if (ctx->chi_cache_bytes < bytes) {
                cudaStreamSynchronize(S);  // the old cache may still be read by an earlier copy
                if (ctx->chi_cache) cudaFree(ctx->chi_cache);
                ctx->chi_cache = nullptr;
                ctx->chi_cache_bytes = 0;
                ctx->chi_key.clear();
                if (cudaMalloc(&ctx->chi_cache, bytes)) return fail(ctx->fail(NEO_ERR_OOM, "mem_oracle: chi cache"));
                ctx->chi_cache_bytes = bytes;
            }
            if (cudaMemcpyAsync(ctx->chi_cache, T, bytes, cudaMemcpyDeviceToDevice, S))
                return fail(ctx->fail(NEO_ERR_CUDA, "mem_oracle: chi cache copy"));
            ctx->chi_key = key;
        }
    }
    cudaError_t ce = cudaSuccess;
    switch (kind) {
        case NEO_MEM_SHOUT_VALUE:
            ce = put(1, 0);
            if (!ce) ce = put(2, 1);
            break;
        case NEO_MEM_SHOUT_ADAPTER:
            ce = put(1, 0);
            if (!ce) rc = eqbits(2, 1);
            break;
        case NEO_MEM_BITNESS:
            for (uint32_t c = 0; c < n_cols && !ce; c++) ce = put(1 + c, c);
            for (uint32_t c = 0; c < n_cols; c++) o->hw.push_back(kload_h(weights + 2 * c));
            if (!ce && n_cols && (o->w.ensure(n_cols) ||
                        cudaMemcpyAsync(o->w.p, weights, n_cols * sizeof(K), cudaMemcpyHostToDevice, S)))
                ce = cudaErrorMemoryAllocation;
            break;
        case NEO_MEM_TWIST_READ:
        case NEO_MEM_TWIST_WRITE: {
            const bool rd = kind == NEO_MEM_TWIST_READ;
            // write stream columns: has_write, inc, wa bits
            const uint32_t c_hw = rd ? 2 + A : 0, c_inc = rd ? 3 + A : 2, c_wa = rd ? 4 + A : 3;
            const uint32_t c_a = rd ? 1 : 1;  // rv (read) or wv (write)
            if (tmp.ensure((size_t)(4 + A) * L)) { ce = cudaErrorMemoryAllocation; break; }
            K* hw = tmp.p;
            K* inc = tmp.p + L;
            K* aa = tmp.p + 2 * L;
            K* terms = tmp.p + 3 * L;
            K* wa = tmp.p + 4 * L;
            ce = cudaMemcpyAsync(hw, col(c_hw), colb, cpk, S);
            if (!ce) ce = cudaMemcpyAsync(inc, col(c_inc), colb, cpk, S);
            if (!ce) ce = cudaMemcpyAsync(aa, col(c_a), colb, cpk, S);
            if (!ce && A) ce = cudaMemcpyAsync(wa, col(c_wa), colb * A, cpk, S);
            if (ce) break;
            inc_terms_kernel<<<ceil_div(L, 256), 256, 0, S>>>(hw, inc, wa, A, dra.p, L, terms);
            NEO_LAUNCHED(ctx);
            const uint32_t nblk = (uint32_t)ceil_div(L, SCAN_BLK);
            DevBuf<K>& sums = o->sums;
            if (sums.ensure(nblk)) { ce = cudaErrorMemoryAllocation; break; }
            scan_sums_kernel<<<nblk, SCAN_T, 0, S>>>(terms, L, sums.p);
            NEO_LAUNCHED(ctx);
            K init_k = init ? kload_h(init) : gl::kzero();
            scan_top_kernel<<<1, SCAN_T, 0, S>>>(sums.p, nblk, init_k);
            NEO_LAUNCHED(ctx);
            // factor 2 = Val_pre − rv  |  wv − Val_pre − inc
            scan_final_kernel<<<nblk, SCAN_T, 0, S>>>(terms, L, sums.p, rd ? 1 : 2, aa, inc, T + 2 * L);
            NEO_LAUNCHED(ctx);
            ce = put(1, 0);  // gate: has_read | has_write
            if (!ce) rc = eqbits(3, rd ? 2 : 3);
        } break;
        case NEO_MEM_VAL_EVAL:
            ce = put(0, 0);
            if (!ce) ce = put(1, 1);
            if (ce) break;
            lt_table_kernel<<<ceil_div(L, 256), 256, 0, S>>>(dpt.p, ell, T + 2 * L);
            NEO_LAUNCHED(ctx);
            rc = eqbits(3, 2);
            break;
        case NEO_MEM_TOTAL_INC:
            ce = put(0, 0);
            if (!ce) ce = put(1, 1);
            if (!ce) rc = eqbits(2, 2);
            break;
        case NEO_MEM_PRODUCT:
            for (uint32_t c = 0; c < n_cols && !ce; c++) ce = put(c, c);
            break;
    }
    if (ce) return fail(ctx->fail(ce == cudaErrorMemoryAllocation ? NEO_ERR_OOM : NEO_ERR_CUDA, "mem_oracle: build", ce));
    if (rc) return fail(rc);
    // claim = Σ over the hypercube = p_0(0) + p_0(1)  (the constructors' sums);
    // a lazy build (the shard: no claim asked for, or claims computed for a
    // group by mem_claims_multi) skips it
    if (!lazy) {
        rc = mem_round_values(o);
        if (rc) return fail(rc);
        o->claim = ell ? gl::kadd(o->hvals[0], o->hvals[1]) : o->hvals[0];
        if (claim_out) {
            claim_out[0] = o->claim.re;
            claim_out[1] = o->claim.im;
        }
        NEO_CK(ctx, ctx_sync(ctx));
    }
    *out = o;
    return NEO_OK;
}

}  // namespace

// True when the oracle's next round has at least one pair (its pending fold
// applied): the rounds that mem_round_launch_multi evaluates.
bool mem_round_multi_ok(const neo_gpu_mem_oracle* o) {
    const uint64_t len = o->pending ? o->len >> 1 : o->len;
    return len >= 2 && o->deg + 1 <= MEM_MAX_DEG + 1;
}

// The next round of n oracles: pending folds, then the values at x = 0..deg
// of oracle i into d_out[i] (device), in one launch and without a host
// sync.  Every oracle must satisfy mem_round_multi_ok; n <= MULTI_MAX.
int mem_round_launch_multi(neo_gpu_ctx* ctx, neo_gpu_mem_oracle* const* os, int n, K* const* d_out,
                           DevBuf<K>& partials) {
    if (n <= 0) return NEO_OK;
    if (n > MULTI_MAX) return ctx->fail(NEO_ERR_UNSUPPORTED, "mem_round_launch_multi: too many claims");
    MultiArgs a{};
    a.n = n;
    uint32_t blocks = 0;
    uint64_t parts = 0;
    for (int i = 0; i < n; i++) {
        neo_gpu_mem_oracle* o = os[i];
        MultiClaim& c = a.c[i];
        c.src = nullptr;
        if (o->pending) {  // the evaluation launch applies the fold (point group 0 writes the tables)
            c.src = o->tab[o->cur].p;
            c.r = o->pending_r;
            o->cur ^= 1;
            o->len >>= 1;
            o->pending = false;
        }
        if (o->len < 2) return ctx->fail(NEO_ERR_INVARIANT, "mem_round_launch_multi: no pairs left");
        c.tab = o->tab[o->cur].p;
        c.len = o->len;
        c.nf = o->nf;
        c.npts = o->deg + 1;
        c.bitness = o->bitness;
        c.w = o->w.p;
        c.blk0 = blocks;
        c.nchunk = o->bitness ? std::max<uint32_t>(1, (uint32_t)ceil_div(o->nf - 1, BIT_CHUNK)) : 1;
        c.nblk = (uint32_t)ceil_div(o->len >> 1, 256) * c.nchunk;
        // points per thread: MX while the pairs fill the GPU, fewer for the
        // small tables of the late rounds (their point groups run in parallel),
        // never more than the claim's points rounded up to a power of two
        const uint64_t pairs = o->len >> 1;
        uint32_t ppt = pairs >= 8192 ? MX : (pairs >= 1024 ? 4 : (pairs >= 256 ? 2 : 1));
        while (ppt > 1 && ppt / 2 >= c.npts) ppt /= 2;
        c.ppt = ppt;
        c.part0 = (uint32_t)parts;
        c.out = d_out[i];
        blocks += c.nblk * (uint32_t)ceil_div(c.npts, c.ppt);
        parts += (uint64_t)c.npts * c.nblk;
    }
    if (parts > 0xFFFFFFFFull) return ctx->fail(NEO_ERR_UNSUPPORTED, "mem_round_launch_multi: too many partials");
    // the claims' tickets sit behind the partials (MULTI_MAX counters in
    // MULTI_TICKET_K entries); they return to zero after every launch, so
    // they are cleared only when the buffer is (re)allocated
    constexpr size_t MULTI_TICKET_K = (MULTI_MAX * sizeof(unsigned int) + sizeof(K) - 1) / sizeof(K);
    const K* before = partials.p;
    const size_t cap_before = partials.cap;
    NEO_CK(ctx, partials.ensure(std::max<uint64_t>(parts, cap_before > MULTI_TICKET_K ? cap_before - MULTI_TICKET_K : 0) +
                                MULTI_TICKET_K));
    unsigned int* tickets = reinterpret_cast<unsigned int*>(partials.p + (partials.cap - MULTI_TICKET_K));
    if (partials.p != before || partials.cap != cap_before)
        NEO_CK(ctx, cudaMemsetAsync(tickets, 0, MULTI_TICKET_K * sizeof(K), ctx->stream));
    for (int i = 0; i < n; i++) a.c[i].ticket = tickets + i;
    a.partials = partials.p;
    mem_multi_eval_kernel<<<blocks, 256, 0, ctx->stream>>>(a);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}



// Claims (sums over the hypercube, p_0(0) + p_0(1)) of n lazily built oracles:
// one multi-claim evaluation of their round 0, one copy and one sync;
// oracles the multi-claim kernel cannot take are evaluated one by one.
int mem_claims_multi(neo_gpu_ctx* ctx, neo_gpu_mem_oracle* const* os, int n, K* claims, DevBuf<K>& partials,
                     DevBuf<K>& d_slots, HostBuf<K>& h_slots) {
    constexpr uint32_t SLOT = MEM_MAX_DEG + 1;
    bool multi = n > 0 && n <= MULTI_MAX;
    for (int i = 0; i < n && multi; i++) multi = mem_round_multi_ok(os[i]) && !os[i]->pending && os[i]->ell > 0;
    if (!multi) {
        for (int i = 0; i < n; i++) {
            neo_gpu_mem_oracle* o = os[i];
            if (int rc = mem_round_values(o)) return rc;
            o->claim = o->ell ? gl::kadd(o->hvals[0], o->hvals[1]) : o->hvals[0];
            claims[i] = o->claim;
        }
        NEO_CK(ctx, ctx_sync(ctx));
        return NEO_OK;
    }
    NEO_CK(ctx, d_slots.ensure((size_t)n * SLOT));
    NEO_CK(ctx, h_slots.ensure((size_t)n * SLOT));
    std::vector<K*> dst(n);
    for (int i = 0; i < n; i++) dst[i] = d_slots.p + (size_t)i * SLOT;
    if (int rc = mem_round_launch_multi(ctx, os, n, dst.data(), partials)) return rc;
    NEO_CK(ctx, cudaMemcpyAsync(h_slots.p, d_slots.p, (size_t)n * SLOT * sizeof(K), cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, ctx_sync(ctx));
    for (int i = 0; i < n; i++) {
        const K* v = h_slots.p + (size_t)i * SLOT;
        os[i]->claim = gl::kadd(v[0], v[1]);
        claims[i] = os[i]->claim;
    }
    return NEO_OK;
}

static int neo_gpu_mem_oracle_create_impl_abi(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point,
                                         uint32_t ell_addr, const uint64_t* r_addr, const uint64_t* init_at_r_addr,
                                         uint32_t n_cols, const uint64_t* cols, const uint64_t* weights,
                                         uint64_t* claim, neo_gpu_mem_oracle** out) {
    return mem_create(ctx, kind, ell, r_point, ell_addr, r_addr, init_at_r_addr, n_cols, cols, false, weights, claim,
                      out);
}
extern "C" int neo_gpu_mem_oracle_create(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point,
                                         uint32_t ell_addr, const uint64_t* r_addr, const uint64_t* init_at_r_addr,
                                         uint32_t n_cols, const uint64_t* cols, const uint64_t* weights,
                                         uint64_t* claim, neo_gpu_mem_oracle** out) { NEO_ABI_GUARD(neo_gpu_mem_oracle_create_impl_abi(ctx, kind, ell, r_point, ell_addr, r_addr, init_at_r_addr, n_cols, cols, weights, claim, out)) }

// Rebuild into *slot when it holds an oracle (its device buffers are kept),
// create one otherwise; columns in device memory.  Fold steps call this every
// step so that no device allocation (a device-wide synchronization for
// cudaFree) happens once the buffers have grown.
int mem_oracle_build_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point, uint32_t ell_addr,
                            const uint64_t* r_addr, const uint64_t* init_at_r_addr, uint32_t n_cols,
                            const uint64_t* d_cols, const uint64_t* weights, uint64_t* claim,
                            neo_gpu_mem_oracle** slot) {
    return mem_create(ctx, kind, ell, r_point, ell_addr, r_addr, init_at_r_addr, n_cols, d_cols, true, weights, claim,
                      slot, true, claim == nullptr);
}

static int neo_gpu_mem_oracle_create_device_impl_abi(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point,
                                                uint32_t ell_addr, const uint64_t* r_addr,
                                                const uint64_t* init_at_r_addr, uint32_t n_cols,
                                                const uint64_t* d_cols, const uint64_t* weights, uint64_t* claim,
                                                neo_gpu_mem_oracle** out) {
    return mem_create(ctx, kind, ell, r_point, ell_addr, r_addr, init_at_r_addr, n_cols, d_cols, true, weights, claim,
                      out);
}
extern "C" int neo_gpu_mem_oracle_create_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_point,
                                                uint32_t ell_addr, const uint64_t* r_addr,
                                                const uint64_t* init_at_r_addr, uint32_t n_cols,
                                                const uint64_t* d_cols, const uint64_t* weights, uint64_t* claim,
                                                neo_gpu_mem_oracle** out) { NEO_ABI_GUARD(neo_gpu_mem_oracle_create_device_impl_abi(ctx, kind, ell, r_point, ell_addr, r_addr, init_at_r_addr, n_cols, d_cols, weights, claim, out)) }

static int neo_gpu_mem_oracle_evals_impl_abi(neo_gpu_mem_oracle* o, const uint64_t* xs, uint32_t nx, uint64_t* ys) {
    if (!o) return NEO_ERR_ARG;
    if ((!xs || !ys) && nx) return o->ctx->fail(NEO_ERR_ARG, "mem_oracle_evals: null buffer");
    cudaSetDevice(o->ctx->device);
    int rc = mem_round_values(o);
    if (rc) return rc;
    for (uint32_t i = 0; i < nx; i++) {
        K y = lagrange_at(o->hvals, kload_h(xs + 2 * i));
        ys[2 * i] = y.re;
        ys[2 * i + 1] = y.im;
    }
    return NEO_OK;
}
extern "C" int neo_gpu_mem_oracle_evals(neo_gpu_mem_oracle* o, const uint64_t* xs, uint32_t nx, uint64_t* ys) { NEO_ABI_GUARD(neo_gpu_mem_oracle_evals_impl_abi(o, xs, nx, ys)) }

static int neo_gpu_mem_oracle_fold_impl_abi(neo_gpu_mem_oracle* o, const uint64_t* r) {
    if (!o) return NEO_ERR_ARG;
    if (!r) return o->ctx->fail(NEO_ERR_ARG, "mem_oracle_fold: null challenge");
    if (o->bit_idx >= o->ell) return NEO_OK;  // no rounds left: ignored, as in the reference
    if (o->pending) {
        // two folds without an evaluation in between: apply the first now
        neo_gpu_ctx* ctx = o->ctx;
        cudaSetDevice(ctx->device);
        uint64_t tot = (o->len >> 1) * o->nf;
        mem_fold_kernel<<<ceil_div(tot, 256), 256, 0, ctx->stream>>>(o->tab[o->cur].p, o->len, o->tab[o->cur ^ 1].p,
                                                                     o->nf, o->pending_r);
        NEO_LAUNCHED(ctx);
        o->cur ^= 1;
        o->len >>= 1;
    }
    o->pending = true;
    o->pending_r = kload_h(r);
    o->bit_idx++;
    return NEO_OK;
}
extern "C" int neo_gpu_mem_oracle_fold(neo_gpu_mem_oracle* o, const uint64_t* r) { NEO_ABI_GUARD(neo_gpu_mem_oracle_fold_impl_abi(o, r)) }

extern "C" uint32_t neo_gpu_mem_oracle_num_rounds(const neo_gpu_mem_oracle* o) { return o ? o->ell - o->bit_idx : 0; }
extern "C" uint32_t neo_gpu_mem_oracle_degree_bound(const neo_gpu_mem_oracle* o) { return o ? o->deg : 0; }

static int neo_gpu_mem_oracle_destroy_impl_abi(neo_gpu_mem_oracle* o) {
    if (!o) return NEO_OK;
    cudaSetDevice(o->ctx->device);
    cudaStreamSynchronize(o->ctx->stream);
    delete o;
    return NEO_OK;
}
extern "C" int neo_gpu_mem_oracle_destroy(neo_gpu_mem_oracle* o) { NEO_ABI_GUARD(neo_gpu_mem_oracle_destroy_impl_abi(o)) }

// AddressLookupOracle weights from device columns: d_rcycle (ell K), d_has
// (2^ell K), d_bits (A columns of 2^ell K), d_table (table_len K).  Writes
// d_w (2^A K) and the claimed sum to *claim (host); synchronizes the stream.
int addr_weights_device(neo_gpu_ctx* ctx, uint32_t ell, const K* d_rcycle, uint32_t A, const K* d_has,
                        const K* d_bits, const K* d_table, uint64_t table_len, K* d_w, K* claim, AddrWs* ws) {
    cudaStream_t S = ctx->stream;
    const uint64_t L = 1ULL << ell, P = 1ULL << A;
    AddrWs local;
    AddrWs& W = ws ? *ws : local;
    DevBuf<K>& chi = W.chi;
    DevBuf<K>& part = W.part;
    DevBuf<K>& out1 = W.out1;
    DevBuf<unsigned long long>& acc = W.acc;
    NEO_CK(ctx, chi.ensure(L));
    NEO_CK(ctx, acc.ensure(4 * P));
    NEO_CK(ctx, cudaMemsetAsync(acc.p, 0, 4 * P * sizeof(unsigned long long), S));
    int rc = launch_chi_table(ctx, d_rcycle, ell, chi.p);
    if (rc) return rc;
    addr_weights_kernel<<<ceil_div(L, 256), 256, 0, S>>>(chi.p, d_has, d_bits, A, L, acc.p, acc.p + 2 * P);
    NEO_LAUNCHED(ctx);
    addr_weights_finish_kernel<<<ceil_div(P, 256), 256, 0, S>>>(acc.p, acc.p + 2 * P, P, d_w);
    NEO_LAUNCHED(ctx);
    const uint64_t n = table_len < P ? table_len : P;
    const uint32_t nb = 148;
    NEO_CK(ctx, part.ensure(nb));
    NEO_CK(ctx, out1.ensure(1));
    dot_kernel<<<nb, 256, 0, S>>>(d_table, d_w, n, part.p);
    NEO_LAUNCHED(ctx);
    mem_reduce_kernel<<<1, 256, 0, S>>>(part.p, nb, out1.p);
    NEO_LAUNCHED(ctx);
    NEO_CK(ctx, ctx_d2h(ctx, claim, out1.p, sizeof(K)));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}

static int neo_gpu_addr_lookup_weights_impl_abi(neo_gpu_ctx* ctx, uint32_t ell, const uint64_t* r_cycle, uint32_t ell_addr,
                                           const uint64_t* has_lookup, const uint64_t* addr_bits,
                                           const uint64_t* table, uint64_t table_len, uint64_t* weights,
                                           uint64_t* claim) {
    if (!ctx) return NEO_ERR_ARG;
    if (!r_cycle || !has_lookup || (!addr_bits && ell_addr) || !weights || !claim || (!table && table_len))
        return ctx->fail(NEO_ERR_ARG, "addr_lookup_weights: null buffer");
    if (ell > 30 || ell_addr > 30) return ctx->fail(NEO_ERR_ARG, "addr_lookup_weights: size");
    cudaSetDevice(ctx->device);
    cudaStream_t S = ctx->stream;
    const uint64_t L = 1ULL << ell, P = 1ULL << ell_addr;
    DevBuf<K> dr, has, bits, w, tab;
    NEO_CK(ctx, dr.alloc(ell ? ell : 1));
    NEO_CK(ctx, has.alloc(L));
    NEO_CK(ctx, bits.alloc((size_t)L * (ell_addr ? ell_addr : 1)));
    NEO_CK(ctx, w.alloc(P));
    NEO_CK(ctx, tab.alloc(table_len ? table_len : 1));
    if (ell) NEO_CK(ctx, cudaMemcpyAsync(dr.p, r_cycle, ell * sizeof(K), cudaMemcpyHostToDevice, S));
    NEO_CK(ctx, cudaMemcpyAsync(has.p, has_lookup, L * sizeof(K), cudaMemcpyHostToDevice, S));
    if (ell_addr) NEO_CK(ctx, cudaMemcpyAsync(bits.p, addr_bits, (size_t)L * ell_addr * sizeof(K), cudaMemcpyHostToDevice, S));
    if (table_len) NEO_CK(ctx, cudaMemcpyAsync(tab.p, table, table_len * sizeof(K), cudaMemcpyHostToDevice, S));
    K cl;
    int rc = addr_weights_device(ctx, ell, dr.p, ell_addr, has.p, bits.p, tab.p, table_len, w.p, &cl, nullptr);
    if (rc) return rc;
    NEO_CK(ctx, ctx_d2h(ctx, weights, w.p, P * sizeof(K)));
    NEO_CK(ctx, ctx_sync(ctx));
    claim[0] = cl.re;
    claim[1] = cl.im;
    return NEO_OK;
}
extern "C" int neo_gpu_addr_lookup_weights(neo_gpu_ctx* ctx, uint32_t ell, const uint64_t* r_cycle, uint32_t ell_addr,
                                           const uint64_t* has_lookup, const uint64_t* addr_bits,
                                           const uint64_t* table, uint64_t table_len, uint64_t* weights,
                                           uint64_t* claim) { NEO_ABI_GUARD(neo_gpu_addr_lookup_weights_impl_abi(ctx, ell, r_cycle, ell_addr, has_lookup, addr_bits, table, table_len, weights, claim)) }

// ===========================================================================
// Twist address-lane oracles (TwistReadCheckAddrOracleSparseTime /
// TwistWriteCheckAddrOracleSparseTime, twist_oracle.rs:1259-1642).
//
// The reference replays a HashMap memory over the time-ordered events every
// round.  Here the events are compacted once into arrays; the memory value a
// query event i sees at address block idx is
//     init_tab[idx] + Σ_{j < i, wa_j >> bit = idx} inc_j·hw_j·wpw_j,
// where init_tab is the initial memory folded on its low address bits (the
// reference's init prefix weights are exactly that fold).  One thread per
// query event sums the earlier writes from shared-memory tiles.  Degree 2:
// values at x = 0, 1, 2 are reduced and interpolated on the host.
// ===========================================================================
namespace {

constexpr int TA_T = 64;

__device__ __forceinline__ uint32_t addr_bits_at(const K* bits, uint64_t L, uint32_t A, uint64_t t) {
    uint32_t a = 0;
    for (uint32_t b = 0; b < A; b++) {
        K v = bits[(uint64_t)b * L + t];
        if (v.re == 1 && v.im == 0) a |= 1u << b;
    }
    return a;
}

// event flags: read kind: has_read | has_write nonzero; write kind: has_write nonzero
__global__ void ta_count_kernel(const K* __restrict__ hr, const K* __restrict__ hw, uint64_t L, uint32_t* __restrict__ counts) {
    __shared__ uint32_t s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    bool f = false;
    if (t < L) f = !gl::kiszero(hw[t]) || (hr && !gl::kiszero(hr[t]));
    unsigned bal = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && bal) atomicAdd(&s_cnt, (uint32_t)__popc(bal));
    __syncthreads();
    if (threadIdx.x == 0) counts[blockIdx.x] = s_cnt;
}

struct TaBuild {
    const K *hr, *rv, *ra, *hw, *inc, *wa, *wv;
    const K* r_cycle;
    uint32_t ell, A;
    uint64_t L;
    const uint32_t* offs;   // exclusive prefix of the per-block counts
    // outputs [E]
    K *eq, *ehr, *erv, *ehw, *einc, *ewv;
    uint32_t *era, *ewa;
};

__global__ void ta_build_kernel(const TaBuild a) {
    __shared__ uint32_t s_warp[TA_T / 32];
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    bool f = false;
    if (t < a.L) f = !gl::kiszero(a.hw[t]) || (a.hr && !gl::kiszero(a.hr[t]));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) s_warp[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; w++) before += s_warp[w];
    before += __popc(bal & ((1u << lane) - 1));
    if (!f) return;
    const uint32_t e = a.offs[blockIdx.x] + before;
    // χ_{r_cycle}(t)
    K chi = gl::kone();
    for (uint32_t i = 0; i < a.ell; i++) {
        K ri = a.r_cycle[i];
        chi = gl::kmul(chi, ((t >> i) & 1) ? ri : gl::ksub(gl::kone(), ri));
    }
    a.eq[e] = chi;
    K hw = a.hw[t];
    a.ehw[e] = hw;
    a.einc[e] = a.inc[t];
    const bool has_w = !gl::kiszero(hw);
    if (a.hr) {
        K hr = a.hr[t];
        a.ehr[e] = hr;
        a.erv[e] = a.rv[t];
        a.era[e] = gl::kiszero(hr) ? 0u : addr_bits_at(a.ra, a.L, a.A, t);
        a.ewa[e] = has_w ? addr_bits_at(a.wa, a.L, a.A, t) : 0u;
    } else {
        a.ewv[e] = a.wv[t];
        a.ewa[e] = addr_bits_at(a.wa, a.L, a.A, t);
    }
}

// one round of the address lane: a block (query block x, event block y) adds
// the earlier writes of event block y to its queries' memory values
struct TaEval {
    int kind;  // 0 read, 1 write
    uint32_t E, bit;
    const K *eq, *hr, *rv, *hw, *inc, *wv, *rpw, *wpw;
    const uint32_t *ra, *wa;
    const K* init_tab;  // folded initial memory, >= 2 entries
    K* partials;        // [3][gridDim.x * gridDim.y]
    K* out;             // the round's values at x = 0, 1, 2 (the last block sums the partials)
    unsigned int* ticket;
};

// grid.x: query events i in tiles of TA_T; grid.y: earlier-event chunks j of
// TA_T.  The contribution is linear in the memory value, so each chunk adds
// w·af(x)·(±its partial memory value) and chunk 0 adds the initial memory and
// the constant terms; the reduction sums all blocks.
__global__ void __launch_bounds__(TA_T) ta_eval_kernel(const TaEval a) {
    __shared__ uint32_t s_key[TA_T];
    __shared__ K s_d[TA_T];
    __shared__ K s_red[3][TA_T / 32];
    const uint32_t i = blockIdx.x * TA_T + threadIdx.x;
    const uint32_t i_end = min(a.E, blockIdx.x * TA_T + TA_T);
    const uint32_t j0 = blockIdx.y * TA_T;
    bool q = false;
    uint32_t addr = 0;
    if (i < a.E) {
        if (a.kind == 0) { q = !gl::kiszero(a.hr[i]); addr = a.ra[i]; }
        else { q = !gl::kiszero(a.hw[i]); addr = a.wa[i]; }
    }
    const uint32_t base = a.bit >= 31 ? 0u : ((addr >> (a.bit + 1)) << 1);
    K v0 = gl::kzero(), v1 = gl::kzero();
    if (q && blockIdx.y == 0) {
        v0 = a.init_tab[base];
        v1 = a.init_tab[base + 1];
    }
    bool any = blockIdx.y == 0;
    if (j0 < i_end) {  // block-uniform: some query of this block has earlier events in the chunk
        const uint32_t j = j0 + threadIdx.x;
        if (j < a.E) {
            // the write event's key (its address block at this bit) and delta
            // inc * has_write * address weight; no write: a key nothing matches
            const K h = a.hw[j];
            const bool w = !gl::kiszero(h);
            s_key[threadIdx.x] = !w ? 0xFFFFFFFFu : (a.bit >= 32 ? 0u : (a.wa[j] >> a.bit));
            s_d[threadIdx.x] = w ? gl::kmul(gl::kmul(a.inc[j], h), a.wpw[j]) : gl::kzero();
        }
        __syncthreads();
        if (q && i > j0) {
            const uint32_t jn = i - j0 < TA_T ? i - j0 : TA_T;
            any = true;
            for (uint32_t u = 0; u < jn; u++) {
                const uint32_t k = s_key[u];
                if (k == base) v0 = gl::kadd(v0, s_d[u]);
                else if (k == base + 1) v1 = gl::kadd(v1, s_d[u]);
            }
        }
    }
    K c[3] = {gl::kzero(), gl::kzero(), gl::kzero()};
    if (q && any) {
        const bool b = a.bit < 32 && ((addr >> a.bit) & 1);
        K w = a.kind == 0 ? gl::kmul(gl::kmul(a.eq[i], a.hr[i]), a.rpw[i]) : gl::kmul(gl::kmul(a.eq[i], a.hw[i]), a.wpw[i]);
        K dv = gl::ksub(v1, v0);
        K vx = v0;
#pragma unroll
        for (int x = 0; x < 3; x++) {
            K af = b ? gl::kfq((uint64_t)x) : gl::kfq(gl::sub(1, (uint64_t)x));
            K term;
            if (blockIdx.y == 0) term = a.kind == 0 ? gl::ksub(vx, a.rv[i]) : gl::ksub(gl::ksub(a.wv[i], vx), a.inc[i]);
            else term = a.kind == 0 ? vx : gl::kneg(vx);
            c[x] = gl::kmul(gl::kmul(w, af), term);
            vx = gl::kadd(vx, dv);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int x = 0; x < 3; x++) {
        K v = c[x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_km(v, o));
        if (lane == 0) s_red[x][warp] = v;
    }
    __syncthreads();
    const uint64_t nb = (uint64_t)gridDim.x * gridDim.y;
    if (threadIdx.x < 3) {
        K s = gl::kzero();
        for (int w = 0; w < TA_T / 32; w++) s = gl::kadd(s, s_red[threadIdx.x][w]);
        a.partials[(uint64_t)threadIdx.x * nb + (uint64_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
    // the last block to finish sums the partials (ticket, no waits)
    __threadfence();
    __syncthreads();
    __shared__ unsigned int s_last;
    if (threadIdx.x == 0) s_last = atomicInc(a.ticket, (unsigned int)(nb - 1)) == nb - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the points x < 3 split over the block's warps, side by side
    for (int x = warp; x < 3; x += TA_T / 32) {
        K v = gl::kzero();
#pragma unroll 4
        for (uint64_t b = lane; b < nb; b += 32) {
            const ulonglong2 u = __ldcg(reinterpret_cast<const ulonglong2*>(a.partials + (uint64_t)x * nb + b));
            v = gl::kadd(v, gl::kmk(u.x, u.y));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = gl::kadd(v, shfl_xor_km(v, o));
        if (lane == 0) a.out[x] = v;
    }
}

// One round's fold of the address lane: threads j < E fold the events'
// address weights by the bound bit, the next `half` fold the initial-memory
// table on its low address bit.
__global__ void ta_fold_kernel(const uint32_t* __restrict__ ra, const uint32_t* __restrict__ wa, K* __restrict__ rpw,
                               K* __restrict__ wpw, uint32_t E, uint32_t bit, K r, int kind, const K* __restrict__ tab,
                               K* __restrict__ tab_out, uint64_t half) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j < E) {
        const K omr = gl::ksub(gl::kone(), r);
        if (kind == 0) rpw[j] = gl::kmul(rpw[j], ((ra[j] >> bit) & 1) ? r : omr);
        wpw[j] = gl::kmul(wpw[j], ((wa[j] >> bit) & 1) ? r : omr);
    } else if (j - E < half) {
        const uint64_t p = j - E;
        tab_out[p] = gl::klerp(tab[2 * p], tab[2 * p + 1], r);
    }
}

__global__ void scatter_init_kernel(const uint64_t* __restrict__ addr, const K* __restrict__ val, uint64_t n,
                                    K* __restrict__ tab) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) tab[addr[i]] = val[i];
}

}  // namespace

struct neo_gpu_twist_addr {
    neo_gpu_ctx* ctx = nullptr;
    int kind = 0;
    uint32_t A = 0, bit = 0, E = 0;
    DevBuf<K> eq, hr, rv, hw, inc, wv, rpw, wpw, tab[2], partials, vals;
    DevBuf<uint32_t> ra, wa;
    DevBuf<unsigned int> ticket;     // ta_eval_kernel's block counter (returns to zero after every launch)
    DevBuf<K> dcols, dr, dv;         // build workspace, kept for reuse
    DevBuf<uint32_t> counts;
    DevBuf<uint64_t> da;
    uint64_t tab_len = 0;
    int cur = 0;
    bool pending = false;
    K pending_r{};
    std::vector<K> hvals;
};

namespace {

int ta_apply_fold(neo_gpu_twist_addr* o) {
    neo_gpu_ctx* ctx = o->ctx;
    cudaStream_t S = ctx->stream;
    // the events' address weights and the initial-memory table, one launch
    const uint64_t half = o->tab_len >> 1;
    const uint64_t n = o->E + half;
    if (n) {
        ta_fold_kernel<<<ceil_div(n, 256), 256, 0, S>>>(o->ra.p, o->wa.p, o->rpw.p, o->wpw.p, o->E, o->bit, o->pending_r,
                                                       o->kind, o->tab[o->cur].p, o->tab[o->cur ^ 1].p, half);
        NEO_LAUNCHED(ctx);
    }
    o->cur ^= 1;
    o->tab_len = half;
    o->bit++;
    o->pending = false;
    return NEO_OK;
}

// The round's values at x = 0, 1, 2 into d_dst (device), without a host sync
// (the pending fold applied first); no events: zeros.
int ta_values_launch(neo_gpu_twist_addr* o, K* d_dst) {
    neo_gpu_ctx* ctx = o->ctx;
    cudaStream_t S = ctx->stream;
    if (o->pending) {
        int rc = ta_apply_fold(o);
        if (rc) return rc;
    }
    if (o->E == 0) {
        NEO_CK(ctx, cudaMemsetAsync(d_dst, 0, 3 * sizeof(K), S));
        return NEO_OK;
    }
    const uint32_t nbx = ceil_div(o->E, TA_T);
    const uint32_t nb = nbx * nbx;
    NEO_CK(ctx, o->partials.ensure((size_t)3 * nb));
    TaEval a;
    a.kind = o->kind;
    a.E = o->E;
    a.bit = o->bit;
    a.eq = o->eq.p; a.hr = o->hr.p; a.rv = o->rv.p; a.hw = o->hw.p; a.inc = o->inc.p; a.wv = o->wv.p;
    a.rpw = o->rpw.p; a.wpw = o->wpw.p; a.ra = o->ra.p; a.wa = o->wa.p;
    a.init_tab = o->tab[o->cur].p;
    a.partials = o->partials.p;
    a.out = d_dst;
    a.ticket = o->ticket.p;
    ta_eval_kernel<<<dim3(nbx, nbx), TA_T, 0, S>>>(a);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}

int ta_values(neo_gpu_twist_addr* o) {
    neo_gpu_ctx* ctx = o->ctx;
    o->hvals.assign(3, gl::kzero());
    if (int rc = ta_values_launch(o, o->vals.p)) return rc;
    NEO_CK(ctx, ctx_d2h(ctx, o->hvals.data(), o->vals.p, 3 * sizeof(K)));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}

int ta_create(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle, uint32_t A, uint64_t n_init,
              const uint64_t* init_addr, const uint64_t* init_val, const uint64_t* cols, bool dev,
              neo_gpu_twist_addr** out, bool reuse = false) {
    if (!ctx || !out) return NEO_ERR_ARG;
    if (!reuse) *out = nullptr;
    if (kind != 0 && kind != 1) return ctx->fail(NEO_ERR_ARG, "twist_addr: kind must be 0 (read) or 1 (write)");
    if (ell > 30 || A > 30 || A == 0) return ctx->fail(NEO_ERR_ARG, "twist_addr: ell / ell_addr out of range");
    if (!cols || (ell && !r_cycle) || (n_init && (!init_addr || !init_val)))
        return ctx->fail(NEO_ERR_ARG, "twist_addr: null buffer");
    for (uint64_t i = 0; i < n_init; i++)
        if (init_addr[i] >> A) return ctx->fail(NEO_ERR_ARG, "twist_addr: init address out of range");
    cudaSetDevice(ctx->device);
    cudaStream_t S = ctx->stream;
    const uint64_t L = 1ULL << ell, P = 1ULL << A;
    const uint32_t n_cols = kind == 0 ? 4 + 2 * A : 3 + A;
    neo_gpu_twist_addr* o = reuse ? *out : nullptr;
    const bool fresh = !o;
    if (fresh) o = new neo_gpu_twist_addr();
    o->ctx = ctx;
    o->kind = kind;
    o->A = A;
    o->bit = 0;
    o->cur = 0;
    o->pending = false;
    auto fail = [&](int rc) {
        if (fresh) delete o;
        return rc;
    };
    DevBuf<K>& dcols = o->dcols;
    DevBuf<K>& dr = o->dr;
    const K* C = reinterpret_cast<const K*>(cols);
    if (!dev) {
        if (dcols.ensure((size_t)n_cols * L)) return fail(ctx->fail(NEO_ERR_OOM, "twist_addr: columns"));
        if (cudaMemcpyAsync(dcols.p, cols, (size_t)n_cols * L * sizeof(K), cudaMemcpyHostToDevice, S))
            return fail(ctx->fail(NEO_ERR_CUDA, "twist_addr: column upload"));
        C = dcols.p;
    }
    if (dr.ensure(ell ? ell : 1)) return fail(ctx->fail(NEO_ERR_OOM, "twist_addr: r"));
    if (ell && cudaMemcpyAsync(dr.p, r_cycle, ell * sizeof(K), cudaMemcpyHostToDevice, S))
        return fail(ctx->fail(NEO_ERR_CUDA, "twist_addr: r upload"));
    TaBuild b{};
    if (kind == 0) {
        b.hr = C; b.rv = C + L; b.ra = C + 2 * L; b.hw = C + (2 + A) * L; b.inc = C + (3 + A) * L; b.wa = C + (4 + A) * L;
    } else {
        b.hw = C; b.wv = C + L; b.inc = C + 2 * L; b.wa = C + 3 * L;
    }
    const uint32_t nblk = ceil_div(L, TA_T);
    DevBuf<uint32_t>& counts = o->counts;
    if (counts.ensure(nblk)) return fail(ctx->fail(NEO_ERR_OOM, "twist_addr: counts"));
    ta_count_kernel<<<nblk, TA_T, 0, S>>>(b.hr, b.hw, L, counts.p);
    NEO_LAUNCHED(ctx);
    std::vector<uint32_t> hc(nblk);
    NEO_CK(ctx, ctx_d2h(ctx, hc.data(), counts.p, nblk * 4));
    NEO_CK(ctx, ctx_sync(ctx));
    uint64_t E = 0;
    for (auto& c : hc) { uint32_t v = c; c = (uint32_t)E; E += v; }
    o->E = (uint32_t)E;
    const size_t ecap = E ? E : 1;
    if (o->eq.ensure(ecap) || o->hr.ensure(ecap) || o->rv.ensure(ecap) || o->hw.ensure(ecap) || o->inc.ensure(ecap) ||
        o->wv.ensure(ecap) || o->rpw.ensure(ecap) || o->wpw.ensure(ecap) ||
        o->ra.ensure(ecap) || o->wa.ensure(ecap) || o->vals.ensure(3) || o->ticket.ensure(1) ||
        o->tab[0].ensure(P + 1) || o->tab[1].ensure(P / 2 + 1))
        return fail(ctx->fail(NEO_ERR_OOM, "twist_addr: event arrays"));
    NEO_CK(ctx, cudaMemsetAsync(o->ticket.p, 0, sizeof(unsigned int), S));
    NEO_CK(ctx, cudaMemcpyAsync(counts.p, hc.data(), nblk * 4, cudaMemcpyHostToDevice, S));
    b.r_cycle = dr.p; b.ell = ell; b.A = A; b.L = L; b.offs = counts.p;
    b.eq = o->eq.p; b.ehr = o->hr.p; b.erv = o->rv.p; b.ehw = o->hw.p; b.einc = o->inc.p; b.ewv = o->wv.p;
    b.era = o->ra.p; b.ewa = o->wa.p;
    NEO_CK(ctx, cudaMemsetAsync(o->ra.p, 0, ecap * 4, S));
    NEO_CK(ctx, cudaMemsetAsync(o->hr.p, 0, ecap * sizeof(K), S));
    NEO_CK(ctx, cudaMemsetAsync(o->wv.p, 0, ecap * sizeof(K), S));
    ta_build_kernel<<<nblk, TA_T, 0, S>>>(b);
    NEO_LAUNCHED(ctx);
    // prefix weights start at one
    std::vector<K> ones(ecap, gl::kone());
    NEO_CK(ctx, cudaMemcpyAsync(o->rpw.p, ones.data(), ecap * sizeof(K), cudaMemcpyHostToDevice, S));
    NEO_CK(ctx, cudaMemcpyAsync(o->wpw.p, ones.data(), ecap * sizeof(K), cudaMemcpyHostToDevice, S));
    // initial memory as a dense table over the 2^A addresses (plus one zero pad)
    NEO_CK(ctx, cudaMemsetAsync(o->tab[0].p, 0, (P + 1) * sizeof(K), S));
    NEO_CK(ctx, cudaMemsetAsync(o->tab[1].p, 0, (P / 2 + 1) * sizeof(K), S));
    if (n_init) {
        DevBuf<uint64_t>& da = o->da;
        DevBuf<K>& dv = o->dv;
        if (da.ensure(n_init) || dv.ensure(n_init)) return fail(ctx->fail(NEO_ERR_OOM, "twist_addr: init"));
        NEO_CK(ctx, cudaMemcpyAsync(da.p, init_addr, n_init * 8, cudaMemcpyHostToDevice, S));
        NEO_CK(ctx, cudaMemcpyAsync(dv.p, init_val, n_init * sizeof(K), cudaMemcpyHostToDevice, S));
        scatter_init_kernel<<<ceil_div(n_init, 256), 256, 0, S>>>(da.p, dv.p, n_init, o->tab[0].p);
        NEO_LAUNCHED(ctx);
    }
    o->tab_len = P;
    NEO_CK(ctx, ctx_sync(ctx));
    *out = o;
    return NEO_OK;
}

}  // namespace

// Rebuild into *slot when it holds an oracle (buffers kept), else create;
// columns in device memory (the fold step's per-step path).
int twist_addr_build_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle, uint32_t ell_addr,
                            uint64_t n_init, const uint64_t* init_addr, const uint64_t* init_val,
                            const uint64_t* d_cols, neo_gpu_twist_addr** slot) {
    return ta_create(ctx, kind, ell, r_cycle, ell_addr, n_init, init_addr, init_val, d_cols, true, slot, true);
}

static int neo_gpu_twist_addr_create_impl_abi(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle,
                                         uint32_t ell_addr, uint64_t n_init, const uint64_t* init_addr,
                                         const uint64_t* init_val, const uint64_t* cols, neo_gpu_twist_addr** out) {
    return ta_create(ctx, kind, ell, r_cycle, ell_addr, n_init, init_addr, init_val, cols, false, out);
}
extern "C" int neo_gpu_twist_addr_create(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle,
                                         uint32_t ell_addr, uint64_t n_init, const uint64_t* init_addr,
                                         const uint64_t* init_val, const uint64_t* cols, neo_gpu_twist_addr** out) { NEO_ABI_GUARD(neo_gpu_twist_addr_create_impl_abi(ctx, kind, ell, r_cycle, ell_addr, n_init, init_addr, init_val, cols, out)) }

static int neo_gpu_twist_addr_create_device_impl_abi(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle,
                                                uint32_t ell_addr, uint64_t n_init, const uint64_t* init_addr,
                                                const uint64_t* init_val, const uint64_t* d_cols,
                                                neo_gpu_twist_addr** out) {
    return ta_create(ctx, kind, ell, r_cycle, ell_addr, n_init, init_addr, init_val, d_cols, true, out);
}
extern "C" int neo_gpu_twist_addr_create_device(neo_gpu_ctx* ctx, int kind, uint32_t ell, const uint64_t* r_cycle,
                                                uint32_t ell_addr, uint64_t n_init, const uint64_t* init_addr,
                                                const uint64_t* init_val, const uint64_t* d_cols,
                                                neo_gpu_twist_addr** out) { NEO_ABI_GUARD(neo_gpu_twist_addr_create_device_impl_abi(ctx, kind, ell, r_cycle, ell_addr, n_init, init_addr, init_val, d_cols, out)) }

// The next round of a Twist address-lane oracle into d_dst[0..3) (device),
// without a host sync; false (nothing launched) once every address bit is
// bound, when the value no longer depends on x.
int ta_round_launch(neo_gpu_twist_addr* o, K* d_dst, bool* launched) {
    *launched = false;
    if (o->bit + (o->pending ? 1 : 0) >= o->A) return NEO_OK;
    cudaSetDevice(o->ctx->device);
    if (int rc = ta_values_launch(o, d_dst)) return rc;
    *launched = true;
    return NEO_OK;
}

static int neo_gpu_twist_addr_evals_impl_abi(neo_gpu_twist_addr* o, const uint64_t* xs, uint32_t nx, uint64_t* ys) {
    if (!o) return NEO_ERR_ARG;
    if ((!xs || !ys) && nx) return o->ctx->fail(NEO_ERR_ARG, "twist_addr_evals: null buffer");
    cudaSetDevice(o->ctx->device);
    int rc = ta_values(o);
    if (rc) return rc;
    for (uint32_t i = 0; i < nx; i++) {
        // after the last round the value does not depend on x (the reference's constant branch)
        K y = o->bit >= o->A ? o->hvals[0] : lagrange_at(o->hvals, kload_h(xs + 2 * i));
        ys[2 * i] = y.re;
        ys[2 * i + 1] = y.im;
    }
    return NEO_OK;
}
extern "C" int neo_gpu_twist_addr_evals(neo_gpu_twist_addr* o, const uint64_t* xs, uint32_t nx, uint64_t* ys) { NEO_ABI_GUARD(neo_gpu_twist_addr_evals_impl_abi(o, xs, nx, ys)) }

static int neo_gpu_twist_addr_fold_impl_abi(neo_gpu_twist_addr* o, const uint64_t* r) {
    if (!o) return NEO_ERR_ARG;
    if (!r) return o->ctx->fail(NEO_ERR_ARG, "twist_addr_fold: null challenge");
    const uint32_t done = o->bit + (o->pending ? 1 : 0);
    if (done >= o->A) return NEO_OK;
    cudaSetDevice(o->ctx->device);
    if (o->pending) {
        int rc = ta_apply_fold(o);
        if (rc) return rc;
    }
    o->pending = true;
    o->pending_r = kload_h(r);
    return NEO_OK;
}
extern "C" int neo_gpu_twist_addr_fold(neo_gpu_twist_addr* o, const uint64_t* r) { NEO_ABI_GUARD(neo_gpu_twist_addr_fold_impl_abi(o, r)) }

extern "C" uint32_t neo_gpu_twist_addr_num_rounds(const neo_gpu_twist_addr* o) {
    return o ? o->A - o->bit - (o->pending ? 1 : 0) : 0;
}
extern "C" uint32_t neo_gpu_twist_addr_degree_bound(const neo_gpu_twist_addr* o) { return o ? 2 : 0; }

static int neo_gpu_twist_addr_destroy_impl_abi(neo_gpu_twist_addr* o) {
    if (!o) return NEO_OK;
    cudaSetDevice(o->ctx->device);
    cudaStreamSynchronize(o->ctx->stream);
    delete o;
    return NEO_OK;
}
extern "C" int neo_gpu_twist_addr_destroy(neo_gpu_twist_addr* o) { NEO_ABI_GUARD(neo_gpu_twist_addr_destroy_impl_abi(o)) }
