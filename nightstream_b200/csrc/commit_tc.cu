// commit_tc.cu -- Ajtai commitment as an exact int8 tensor-core GEMM (tcgen05).
//
// c_i(X) = sum_j M[i][j](X) z_j(X) mod Phi_81 (crates/neo-ajtai/src/commit.rs:679-744).
// Phi_81 divides X^81 - 1, so the product is taken mod X^81 - 1 (a length-81
// cyclic convolution whose matrix entries are the raw PP coefficients) and
// folded back with X^54 = -X^27 - 1.  As a GEMM:
//
//   D[(i,l)][(v,r)] = sum_{j, s<64} A[(i,l)][(j,s)] * B[(v,r)][(j,s)]
//   A[(i,l)][(j,s)] = byte l of M[i][j][s]  (u8; 0 for s >= 54)
//   B[(v,r)][(j,s)] = z_{v,j}[(r - s) mod 81] (s8; z[x] = 0 for x >= 54)
//   c'_{v,i}[r] = sum_l 2^(8l) D[(i,l)][(v,r)]  (mod q), r < 81
//
// M = 128 = kappa * 8 rows, K = 64 m (s padded to 64 so one 128-byte K block
// holds exactly two columns j), N = 81 per vector.  Accumulation is int32 in
// TMEM; a CTA covers at most 512 K blocks, so |D| <= 255*128*65536 < 2^31 for
// any int8 digit: no overflow.  CTAs split K and groups of NV vectors; a second
// kernel sums the int32 partials, recombines limbs mod q and folds 81 -> 54.
//
// A tiles are stored in HBM already in the 128B-swizzled K-major UMMA layout
// (16 KB per K block, contiguous) and fetched with one cp.async.bulk each.
//
// B is never materialised row by row.  With F_{v,j}[w] = z_{v,j}[(80 - w) mod 81]
// (160 bytes per column, precomputed) the B row of output r is the window
// F[r' + s], s < 64, with r' = 80 - r.  Writing r' = 16a + 8h + b, that window
// is the 16-byte-aligned chunks a + k (k < 4) of the phase sequence
// G_p[x] = F[x + p], p = 8h + b.  So the builders write, per column, the 16
// phase sequences as 9 chunks of 16 bytes laid out [chunk][h][v][b] (9 KB),
// and a no-swizzle K-major descriptor with 8-row-group stride 128 B and
// K-chunk stride NV*256 B walks all rows (a, h, v, b) of all NV vectors: row
// group g = (2a + h) NV + v sits at g*128 and its K chunk k at
// (a + k) NV 256 = g-part + k*LBO.  Rows r' < 88 per vector (44 groups,
// N = 256 + 96); r' in [81, 88) are computed and discarded.
#include "internal.cuh"

namespace {

constexpr int TC_NV = 4;                    // vectors per CTA
constexpr int TC_NPAD = 352;                // MMA N total: 44 groups of 8 rows, r' < 88 per vector
constexpr int TC_N0 = 256, TC_N1 = TC_NPAD - 256;  // two MMAs per K step (N = 256, 96)
constexpr int TC_ASTAGES = 6;               // A tiles + F sequences ring (bulk copies run ahead)
constexpr int TC_BSTAGES = 4;               // B phase buffers ring (built by threads, overlaps MMA)
constexpr int TC_A_BYTES = 128 * 128;       // 16 KB
constexpr int TC_BCHUNKS = 9;               // 16-byte K chunks per column: a + k, a <= 5, k < 4
constexpr int TC_BCOL_BYTES = TC_BCHUNKS * TC_NV * 256;  // [chunk][h][v][b][16 B] = 9 KB per column
constexpr int TC_B_BYTES = 2 * TC_BCOL_BYTES;            // two columns per K block: 18 KB
constexpr int TC_BLBO = TC_NV * 256;        // K-direction core-matrix stride (bytes)
constexpr int TC_BSBO = 128;                // N-direction 8-row-group stride (bytes)
constexpr int TC_FBYTES = 160;              // F sequence length (10 x 16 B)
constexpr int TC_F_STAGE = TC_NV * 2 * TC_FBYTES;  // NV x 2 columns x 160 B
constexpr int TC_SMEM_BYTES = TC_ASTAGES * (TC_A_BYTES + TC_F_STAGE) + TC_BSTAGES * TC_B_BYTES;
constexpr int TC_BUILDERS = 256;            // 8 builder warps
constexpr int TC_THREADS = 64 + TC_BUILDERS;  // warp0 producer, warp1 MMA, warps2-9 B build (2-5 epilogue)
constexpr int TC_MAX_KB = 512;              // K blocks per CTA (int32 overflow bound)
constexpr uint32_t TC_SPIN_LIMIT = 1u << 22;       // wait attempts (each suspends at most a hardware limit)
constexpr uint64_t TC_WAIT_NS = 500ull * 1000 * 1000;  // 0.5 s of global time per wait

static_assert(TC_B_BYTES % 1024 == 0 && TC_A_BYTES % 1024 == 0, "stage buffers stay 1024-byte aligned");
static_assert(TC_SMEM_BYTES + 1024 + 256 <= 232448, "shared memory budget");
static_assert(TC_NPAD % 16 == 0 && TC_N1 % 16 == 0 && TC_N1 >= 16, "MMA N constraints (M=128)");
static_assert(TC_N0 == 32 * 8, "the first MMA covers row groups 0..31");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// bounded wait on phase parity; false on timeout.  mbarrier.try_wait suspends
// the thread until the phase completes or a hardware time limit passes, so a
// waiting warp does not keep polling shared memory; the wait gives up after
// TC_WAIT_NS of global time or TC_SPIN_LIMIT attempts, whichever comes first.
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    uint64_t t0 = 0;
    for (uint32_t it = 0; it < TC_SPIN_LIMIT; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        const uint64_t t = globaltimer_ns();
        if (it == 0)
            t0 = t;
        else if (t - t0 > TC_WAIT_NS)
            return false;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// UMMA shared-memory descriptor: K-major, 128B swizzle, 8-row atoms 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                           // leading byte offset (unused for SW128 K-major)
    d |= (uint64_t)(1024 >> 4) << 32;                 // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                           // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                           // layout: SWIZZLE_128B
    return d;
}

// UMMA shared-memory descriptor: K-major, no swizzle: 8-row x 16-byte core
// matrices, LBO between core matrices along K, SBO between 8-row groups.
__device__ __forceinline__ uint64_t ns_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((TC_BLBO >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((TC_BSBO >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100); layout bits 61-63 = 0: no swizzle
    return d;
}

// instruction descriptor: kind::i8, D = s32, A = u8 (K-major), B = s8 (K-major), M = 128
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
    return (2u << 4)            // c_format = S32
           | (0u << 7)          // a_format = unsigned 8-bit
           | (1u << 10)         // b_format = signed 8-bit
           | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ---------------------------------------------------------------------------
// prep: PP -> pre-swizzled u8 limb tiles  PPL[kb][row][128 B]
// ---------------------------------------------------------------------------
// One CTA per K block kb (columns 2kb, 2kb+1): thread (i, jj, g) loads the 8
// coefficients s = 8g..8g+7 of M[i][2kb+jj] (one coalesced 64-byte run),
// splits them into 8 byte planes l and stores each 8-byte piece at row
// (i, l), K offset 64 jj + 8g of the swizzled tile in shared memory; the
// 16 KB tile then goes out as 1024 contiguous 16-byte stores.
__global__ void __launch_bounds__(256) pp_limbs_kernel(const uint64_t* __restrict__ pp, uint32_t kappa, uint64_t m,
                                                       uint8_t* __restrict__ ppl) {
    __shared__ __align__(16) uint8_t tile[TC_A_BYTES];
    const uint64_t kb = blockIdx.x;
    const uint32_t t = threadIdx.x;
    const uint32_t i = t >> 4, jj = (t >> 3) & 1, g = t & 7;
    uint64_t w[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const uint32_t s_ = g * 8 + e;
        w[e] = (i < kappa && s_ < NEO_D) ? pp[((uint64_t)i * m + kb * 2 + jj) * NEO_D + s_] : 0;
    }
    const uint32_t k = jj * 64 + g * 8;  // K byte offset of this 8-byte piece
#pragma unroll
    for (int l = 0; l < 8; l++) {
        uint64_t v = 0;
#pragma unroll
        for (int e = 0; e < 8; e++) v |= ((w[e] >> (8 * l)) & 0xFFull) << (8 * e);
        const uint32_t row = i * 8 + l;
        *reinterpret_cast<uint64_t*>(tile + row * 128 + ((((k >> 4) ^ (row & 7)) << 4) | (k & 15))) = v;
    }
    __syncthreads();
    uint4* dst = reinterpret_cast<uint4*>(ppl + kb * TC_A_BYTES);
    const uint4* src = reinterpret_cast<const uint4*>(tile);
#pragma unroll
    for (int q = 0; q < TC_A_BYTES / 16 / 256; q++) dst[t + 256 * q] = src[t + 256 * q];
}

// prep: F[v][j][w] = z_{v,j}[(80 - w) mod 81] (0 for indices >= 54), w < 160
__global__ void f_seq_kernel(const int8_t* __restrict__ digits, uint32_t n_vec, uint64_t m, uint8_t* __restrict__ F) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (tid >= (uint64_t)n_vec * m) return;
    const uint64_t v = tid / m, j = tid % m;
    int8_t z[NEO_D];
    const int8_t* zv = digits + v * NEO_D * m + j;
#pragma unroll
    for (int x = 0; x < NEO_D; x++) z[x] = zv[(uint64_t)x * m];
    uint32_t w32[TC_FBYTES / 4];
#pragma unroll
    for (int q = 0; q < TC_FBYTES / 4; q++) {
        uint32_t word = 0;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            int w = q * 4 + b;
            int x = w <= 80 ? 80 - w : 161 - w;
            uint8_t byte = (x >= 0 && x < NEO_D) ? (uint8_t)z[x] : 0;
            word |= (uint32_t)byte << (8 * b);
        }
        w32[q] = word;
    }
    uint4* dst = reinterpret_cast<uint4*>(F + tid * TC_FBYTES);
#pragma unroll
    for (int q = 0; q < TC_FBYTES / 16; q++) dst[q] = make_uint4(w32[4 * q], w32[4 * q + 1], w32[4 * q + 2], w32[4 * q + 3]);
}

// ---------------------------------------------------------------------------
// main GEMM kernel
// ---------------------------------------------------------------------------
struct TcArgs {
    const uint8_t* ppl;     // pre-swizzled limb tiles
    const uint8_t* F;       // [n_vec][m][144]
    int32_t* partial;       // [n_cta][128][TC_NPAD]
    uint32_t* err;          // error flag (timeouts)
    uint64_t m;
    uint32_t n_vec, n_groups, n_ksplit, kb_per_cta, n_kb;
};

__global__ void __launch_bounds__(TC_THREADS, 1) commit_tc_kernel(const TcArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-align the tile buffers (dynamic smem base alignment is not guaranteed)
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;                                        // [ASTAGES][16 KB]
    uint8_t* sB = sA + TC_ASTAGES * TC_A_BYTES;                // [BSTAGES][18 KB]
    uint8_t* sF = sB + TC_BSTAGES * TC_B_BYTES;                // [ASTAGES][1280 B]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sF + TC_ASTAGES * TC_F_STAGE);
    uint64_t* full_a = bars;                                   // [ASTAGES] A tile + F landed
    uint64_t* empty_a = bars + TC_ASTAGES;                     // [ASTAGES] MMAs done reading the A tile
    uint64_t* full_b = bars + 2 * TC_ASTAGES;                  // [BSTAGES] B tile built
    uint64_t* empty_b = full_b + TC_BSTAGES;                   // [BSTAGES] MMAs done reading the B tile
    uint64_t* done = empty_b + TC_BSTAGES;                     // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    __shared__ int s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t cta = blockIdx.x;
    const uint32_t group = cta % a.n_groups, ks = cta / a.n_groups;
    const uint32_t kb0 = ks * a.kb_per_cta;
    const uint32_t kb1 = min(a.n_kb, kb0 + a.kb_per_cta);
    const uint32_t nkb = kb1 > kb0 ? kb1 - kb0 : 0;
    const uint32_t nvalid = min((uint32_t)TC_NV, a.n_vec - group * TC_NV);  // vectors of this group

    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int s = 0; s < TC_ASTAGES; s++) {
            mbar_init(&full_a[s], 1);
            mbar_init(&empty_a[s], 1);
        }
        for (int s = 0; s < TC_BSTAGES; s++) {
            mbar_init(&full_b[s], TC_BUILDERS / 32);
            mbar_init(&empty_b[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---- producer: A tiles and F sequences ----
        if (lane == 0) {
            for (uint32_t it = 0; it < nkb; it++) {
                const int s = it % TC_ASTAGES;
                const uint32_t ph = (it / TC_ASTAGES) & 1;
                if (it >= TC_ASTAGES && !mbar_wait(&empty_a[s], ph ^ 1)) { atomicOr(a.err, 1u); s_abort = 1; break; }
                if (s_abort) break;
                const uint64_t kb = kb0 + it;
                mbar_expect_tx(&full_a[s], TC_A_BYTES + nvalid * 2 * TC_FBYTES);
                bulk_g2s(sA + s * TC_A_BYTES, a.ppl + kb * TC_A_BYTES, TC_A_BYTES, &full_a[s]);
                // F sequences of columns 2kb, 2kb+1 for each vector of the group (288 contiguous bytes)
                for (uint32_t vl = 0; vl < nvalid; vl++)
                    bulk_g2s(sF + s * TC_F_STAGE + vl * 2 * TC_FBYTES,
                             a.F + ((uint64_t)(group * TC_NV + vl) * a.m + kb * 2) * TC_FBYTES, 2 * TC_FBYTES, &full_a[s]);
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t id0 = idesc_i8(TC_N0), id1 = idesc_i8(TC_N1);
            for (uint32_t it = 0; it < nkb; it++) {
                const int sa = it % TC_ASTAGES, sb = it % TC_BSTAGES;
                if (!mbar_wait(&full_a[sa], (it / TC_ASTAGES) & 1) || !mbar_wait(&full_b[sb], (it / TC_BSTAGES) & 1)) {
                    atomicOr(a.err, 2u);
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a0 = smem_u32(sA + sa * TC_A_BYTES), b0 = smem_u32(sB + sb * TC_B_BYTES);
#pragma unroll
                for (int k = 0; k < 4; k++) {  // 4 x 32-byte K steps: column k/2, s in [32(k%2), 32(k%2)+32)
                    const uint64_t ad = sw128_desc(a0 + 32 * k);
                    const uint32_t acc = (it > 0 || k > 0) ? 1u : 0u;
                    const uint32_t bcol = b0 + (k >> 1) * TC_BCOL_BYTES + (k & 1) * 2 * TC_BLBO;
                    mma_i8(tmem, ad, ns_desc(bcol), id0, acc);
                    mma_i8(tmem + TC_N0, ad, ns_desc(bcol + 32 * TC_BSBO), id1, acc);
                }
                mma_commit(&empty_a[sa]);  // tiles free once these MMAs complete
                mma_commit(&empty_b[sb]);
            }
            mma_commit(done);
        }
    } else {
        // ---- B builders (warps 2..9) ----
        // thread (part, column jj, vector vl, phase p = 8h + b) writes chunks c of
        // G_p: chunk c = F[16c + p, 16c + p + 16) at [jj][c][h][vl][b]; part 0 the
        // chunks 0..4, part 1 the chunks 5..8 (warp-uniform)
        const int bt = threadIdx.x - 64;
        const int p = bt & 15, vl = (bt >> 4) & 3, jj = (bt >> 6) & 1, part = bt >> 7;
        for (uint32_t it = 0; it < nkb; it++) {
            const int sa = it % TC_ASTAGES, sb = it % TC_BSTAGES;
            // F of this K block has landed, and the MMAs of K block it - BSTAGES released the B buffer;
            // lane 0 waits for the warp, so every exit from this loop is warp-uniform
            uint32_t st = 0;  // 0 go, 1 timed out, 2 another role aborted
            if (lane == 0) {
                if (!mbar_wait(&full_a[sa], (it / TC_ASTAGES) & 1) ||
                    (it >= TC_BSTAGES && !mbar_wait(&empty_b[sb], ((it / TC_BSTAGES) & 1) ^ 1)))
                    st = 1;
                else if (s_abort)
                    st = 2;
            }
            st = __shfl_sync(0xffffffffu, st, 0);
            if (st == 1 && lane == 0) {
                atomicOr(a.err, 4u);
                s_abort = 1;
            }
            if (st) break;
            uint8_t* dstB = sB + sb * TC_B_BYTES;
            const uint8_t* srcF = sF + sa * TC_F_STAGE;
            if ((uint32_t)vl < nvalid) {
                const int c0 = part ? 5 : 0;
                const int o = 16 * c0 + p;  // first F byte of this thread's chunks
                const uint32_t* src = reinterpret_cast<const uint32_t*>(srcF + (vl * 2 + jj) * TC_FBYTES + (o & ~3));
                const uint32_t sh = 8 * (o & 3);
                uint8_t* dst = dstB + jj * TC_BCOL_BYTES + c0 * TC_BLBO + (p >> 3) * (TC_NV * 128) + vl * 128 + (p & 7) * 16;
                uint32_t w[21];
                if (part == 0) {  // 5 chunks: words [o/4, o/4 + 21) <= byte 96 of the 160-byte F
#pragma unroll
                    for (int q = 0; q < 21; q++) w[q] = src[q];
#pragma unroll
                    for (int c = 0; c < 5; c++)
                        *reinterpret_cast<uint4*>(dst + c * TC_BLBO) =
                            make_uint4(__funnelshift_r(w[4 * c], w[4 * c + 1], sh), __funnelshift_r(w[4 * c + 1], w[4 * c + 2], sh),
                                       __funnelshift_r(w[4 * c + 2], w[4 * c + 3], sh), __funnelshift_r(w[4 * c + 3], w[4 * c + 4], sh));
                } else {  // 4 chunks: words [o/4, o/4 + 17) end exactly at byte 160
#pragma unroll
                    for (int q = 0; q < 17; q++) w[q] = src[q];
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        *reinterpret_cast<uint4*>(dst + c * TC_BLBO) =
                            make_uint4(__funnelshift_r(w[4 * c], w[4 * c + 1], sh), __funnelshift_r(w[4 * c + 1], w[4 * c + 2], sh),
                                       __funnelshift_r(w[4 * c + 2], w[4 * c + 3], sh), __funnelshift_r(w[4 * c + 3], w[4 * c + 4], sh));
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&full_b[sb]);
        }
        // ---- epilogue (warps 2..5 cover TMEM lane groups 2, 3, 0, 1): TMEM -> int32 partials ----
        uint32_t okw = 0;  // lane 0 waits for the warp
        if (lane == 0) okw = (nkb > 0 && !s_abort && mbar_wait(done, 0)) ? 1u : 0u;
        const bool ok = __shfl_sync(0xffffffffu, okw, 0) != 0;
        if (nkb > 0 && !ok && warp < 6) atomicOr(a.err, 8u);
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int lg = warp & 3;  // TMEM lane group this warp may access
        const int row = lg * 32 + lane;
        int32_t* dst = a.partial + ((uint64_t)cta * 128 + row) * TC_NPAD;
        for (int c0 = 0; c0 < (warp < 6 ? TC_NPAD : 0); c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (ok) {
#pragma unroll
                for (int q = 0; q < 16; q += 4)
                    *reinterpret_cast<int4*>(dst + c0 + q) = make_int4((int)v[q], (int)v[q + 1], (int)v[q + 2], (int)v[q + 3]);
            } else {
#pragma unroll
                for (int q = 0; q < 16; q += 4) *reinterpret_cast<int4*>(dst + c0 + q) = make_int4(0, 0, 0, 0);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// c'_{v,i}[r] = sum_{ks} sum_l 2^(8l) D[ks][(i,l)][(v,r)] mod q, then fold 81 -> 54.
// One block per (vector group, i): thread (col, half) sums the int32 partials
// of TMEM column col over its half of the K splits for the 8 limb rows
// (reads coalesced along the 352 columns), the halves meet in shared memory,
// then each column is recombined mod q, mapped back to (v, r) and folded.
constexpr int RED_THREADS = TC_NPAD * 2;
__global__ void __launch_bounds__(RED_THREADS) commit_tc_reduce_kernel(const int32_t* __restrict__ partial,
                                                                       uint32_t n_groups, uint32_t n_ksplit,
                                                                       uint32_t kappa, uint32_t n_vec,
                                                                       uint64_t* __restrict__ out) {
    const uint32_t group = blockIdx.x / kappa, i = blockIdx.x % kappa;
    const int col = threadIdx.x % TC_NPAD, half = threadIdx.x / TC_NPAD;
    __shared__ int64_t s_acc[TC_NPAD][8];
    __shared__ uint64_t s_c[TC_NV][81];
    int64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const uint32_t ks0 = half ? n_ksplit / 2 : 0, ks1 = half ? n_ksplit : n_ksplit / 2;
    for (uint32_t ks = ks0; ks < ks1; ks++) {
        const int32_t* p = partial + ((uint64_t)(ks * n_groups + group) * 128 + i * 8) * TC_NPAD + col;
#pragma unroll
        for (int l = 0; l < 8; l++) acc[l] += p[(uint64_t)l * TC_NPAD];
    }
    if (half) {
#pragma unroll
        for (int l = 0; l < 8; l++) s_acc[col][l] = acc[l];
    }
    __syncthreads();
    if (!half) {
        uint64_t c = 0;
#pragma unroll
        for (int l = 0; l < 8; l++) c = gl::add(c, gl::mul(gl::from_i64(acc[l] + s_acc[col][l]), 1ULL << (8 * l)));
        // column -> row group g = (2a + h) NV + v, row b; r' = 16a + 8h + b, r = 80 - r'
        const int g = col >> 3, b = col & 7;
        const int v = g % TC_NV, h = (g / TC_NV) & 1, a = g / (2 * TC_NV);
        const int rp = 16 * a + 8 * h + b;
        if (rp <= 80) s_c[v][80 - rp] = c;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < TC_NV * NEO_D; x += blockDim.x) {
        const int v = x / NEO_D, r = x % NEO_D;
        const uint32_t vg = group * TC_NV + v;
        if (vg < n_vec)
            out[((uint64_t)vg * kappa + i) * NEO_D + r] = gl::sub(s_c[v][r], r >= 27 ? s_c[v][r + 27] : s_c[v][r + 54]);
    }
}

// ---------------------------------------------------------------------------
// Small-digit form: the product taken mod Phi_81 directly.
//
// For digits |z| <= 63 the rotation matrix of z mod Phi_81 itself fits int8:
// [X^r] X^s z(X) mod Phi_81 = z[r-s] - z[r+27-s]                 (r >= 27)
//                             z[r-s] - z[r+54-s] + z[r+81-s]      (r < 27)
// (X^54 = -X^27 - 1 and X^81 = 1 mod Phi_81; z[x] = 0 outside [0, 54)), and
// at most two of the terms are nonzero for any (r, s).  With r' = 58 - r for
// the rows r >= 27 and r' = 31 - r for the rows r < 27 (r' < 32, rows r' < 5
// computed and discarded), row r is the window [r', r' + 64) of one of two
// sequences per (vector, column):
//   H_0[w] = z[58 - w] - z[85 - w],   H_1[w] = z[31 - w] - z[85 - w] + z[112 - w].
// So the B operand keeps the phase-sequence layout of the cyclic form with
// 64 rows per vector instead of 88: N = 64 NV, one MMA per 32-byte K step
// (A read once), 1.40x the algorithmic MACs instead of 1.93x, and the output
// needs no 81 -> 54 fold.  Row groups g = ((2a + h) 2 + seq) NV + v, r' =
// 16a + 8h + b; phase chunks [chunk][h][seq][v][b][16 B], chunk < 5.
constexpr int P8_HSEQ = 112;            // bytes per window sequence (w < 95 used)
constexpr int P8_FBYTES = 2 * P8_HSEQ;  // both sequences of one (vector, column)

template <int NV>
struct P8 {
    static constexpr int NPAD = 64 * NV;        // MMA N
    static constexpr int LBO = 4 * NV * 128;    // K-direction core-matrix stride
    static constexpr int BCOL = 5 * LBO;        // B bytes per column
    static constexpr int B_BYTES = 2 * BCOL;    // two columns per K block
    static constexpr int F_STAGE = NV * 2 * P8_FBYTES;
    // (column, vector, seq, phase pair) for NV <= 4; at least the 4 epilogue warps
    static constexpr int BUILDERS = 128;
    static_assert(NV <= 4, "one builder thread per (column, vector, seq, phase pair)");
    static constexpr int THREADS = 64 + BUILDERS;
    // groups of 4 vectors run two CTAs per SM (3 A stages, 2 B buffers each):
    // while one waits on its rings the other issues MMAs (0.47 instead of
    // 0.52 ms for 12 planes at m = 2^16); a single vector keeps one CTA with
    // deeper rings
    static constexpr int CTAS = NV == 4 ? 2 : 1;
    static constexpr int ASTAGES = CTAS == 2 ? 3 : 6, BSTAGES = CTAS == 2 ? 2 : 4;
    static constexpr int SMEM = ASTAGES * (TC_A_BYTES + F_STAGE) + BSTAGES * B_BYTES;
    static constexpr uint32_t TMEM_COLS = NPAD <= 64 ? 64 : (NPAD <= 128 ? 128 : 256);
    static_assert(NPAD <= 256 && NPAD % 16 == 0, "one MMA per K step (M = 128: N <= 256, N % 16 == 0)");
    static_assert(B_BYTES % 1024 == 0, "B stages stay 1024-byte aligned");
    static_assert(SMEM + 1024 + 256 <= 232448 / CTAS - 1024 * (CTAS - 1), "shared memory budget");
    static_assert(TMEM_COLS * CTAS <= 512, "TMEM columns of the resident CTAs");
};

__device__ __forceinline__ uint64_t ns_desc_lbo(uint32_t saddr, uint32_t lbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((TC_BSBO >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// z[x], 0 outside [0, 54) (x is a compile-time constant after unrolling)
__device__ __forceinline__ int zat(const int (&z)[NEO_D], int x) { return (x >= 0 && x < NEO_D) ? z[x] : 0; }

// prep: the two window sequences of every (vector, column); a digit pair whose
// window entry leaves int8 sets bit 16 of *err (the caller then takes the
// cyclic form, or reports the error).  A block's 128 outputs are contiguous
// (28 KB), so each thread writes its 224 bytes into shared memory (pitch 240 B:
// an odd count of 16-byte chunks keeps a store phase on eight bank groups) and
// the block copies them out with consecutive 16-byte stores.
constexpr int P8_SEQ_THREADS = 128;
constexpr int P8_SEQ_PITCH = P8_FBYTES + 16;
__global__ void __launch_bounds__(P8_SEQ_THREADS) p8_seq_kernel(const int8_t* __restrict__ digits, uint32_t n_vec,
                                                                uint64_t m, uint8_t* __restrict__ F,
                                                                uint32_t* __restrict__ err) {
    __shared__ __align__(16) uint8_t s_out[P8_SEQ_THREADS * P8_SEQ_PITCH];
    const uint64_t total = (uint64_t)n_vec * m;
    const uint64_t base = (uint64_t)blockIdx.x * P8_SEQ_THREADS;
    const uint64_t tid = base + threadIdx.x;
    if (tid < total) {
        const uint64_t v = tid / m, j = tid % m;
        int z[NEO_D];
        const int8_t* zv = digits + v * NEO_D * m + j;
#pragma unroll
        for (int x = 0; x < NEO_D; x++) z[x] = zv[(uint64_t)x * m];
        uint4* dst = reinterpret_cast<uint4*>(s_out + threadIdx.x * P8_SEQ_PITCH);
        bool bad = false;
#pragma unroll
        for (int seq = 0; seq < 2; seq++) {
#pragma unroll
            for (int q = 0; q < P8_HSEQ / 16; q++) {
                uint32_t w4[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    uint32_t word = 0;
#pragma unroll
                    for (int b = 0; b < 4; b++) {
                        const int w = q * 16 + e * 4 + b;
                        const int h = seq == 0 ? zat(z, 58 - w) - zat(z, 85 - w)
                                               : zat(z, 31 - w) - zat(z, 85 - w) + zat(z, 112 - w);
                        bad |= h < -128 || h > 127;
                        word |= (uint32_t)(uint8_t)(int8_t)h << (8 * b);
                    }
                    w4[e] = word;
                }
                dst[seq * (P8_HSEQ / 16) + q] = make_uint4(w4[0], w4[1], w4[2], w4[3]);
            }
        }
        if (bad) atomicOr(err, 1u << 16);
    }
    __syncthreads();
    const uint32_t cnt = (uint32_t)min((uint64_t)P8_SEQ_THREADS, total - base);
    constexpr uint32_t CH = P8_FBYTES / 16;  // 14 chunks per output
    uint4* out = reinterpret_cast<uint4*>(F + base * P8_FBYTES);
    for (uint32_t k = threadIdx.x; k < cnt * CH; k += P8_SEQ_THREADS)
        out[k] = *reinterpret_cast<const uint4*>(s_out + (k / CH) * P8_SEQ_PITCH + (k % CH) * 16);
}

template <int NV>
__global__ void __launch_bounds__(P8<NV>::THREADS, P8<NV>::CTAS) commit_p8_kernel(const TcArgs a) {
    using S = P8<NV>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;                                  // [ASTAGES][16 KB]
    uint8_t* sB = sA + S::ASTAGES * TC_A_BYTES;          // [BSTAGES][B_BYTES]
    uint8_t* sF = sB + S::BSTAGES * S::B_BYTES;          // [ASTAGES][F_STAGE]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sF + S::ASTAGES * S::F_STAGE);
    uint64_t* full_a = bars;
    uint64_t* empty_a = bars + S::ASTAGES;
    uint64_t* full_b = bars + 2 * S::ASTAGES;
    uint64_t* empty_b = full_b + S::BSTAGES;
    uint64_t* done = empty_b + S::BSTAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    __shared__ int s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t cta = blockIdx.x;
    const uint32_t group = cta % a.n_groups, ks = cta / a.n_groups;
    const uint32_t kb0 = ks * a.kb_per_cta;
    const uint32_t kb1 = min(a.n_kb, kb0 + a.kb_per_cta);
    const uint32_t nkb = kb1 > kb0 ? kb1 - kb0 : 0;
    const uint32_t nvalid = min((uint32_t)NV, a.n_vec - group * NV);

    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int s = 0; s < S::ASTAGES; s++) {
            mbar_init(&full_a[s], 1);
            mbar_init(&empty_a[s], 1);
        }
        for (int s = 0; s < S::BSTAGES; s++) {
            mbar_init(&full_b[s], S::BUILDERS / 32);
            mbar_init(&empty_b[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "n"(S::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---- producer: A tiles and window sequences ----
        if (lane == 0) {
            for (uint32_t it = 0; it < nkb; it++) {
                const int s = it % S::ASTAGES;
                const uint32_t ph = (it / S::ASTAGES) & 1;
                if (it >= S::ASTAGES && !mbar_wait(&empty_a[s], ph ^ 1)) { atomicOr(a.err, 1u); s_abort = 1; break; }
                if (s_abort) break;
                const uint64_t kb = kb0 + it;
                mbar_expect_tx(&full_a[s], TC_A_BYTES + nvalid * 2 * P8_FBYTES);
                bulk_g2s(sA + s * TC_A_BYTES, a.ppl + kb * TC_A_BYTES, TC_A_BYTES, &full_a[s]);
                for (uint32_t vl = 0; vl < nvalid; vl++)  // columns 2kb, 2kb+1 of vector vl: 448 contiguous bytes
                    bulk_g2s(sF + s * S::F_STAGE + vl * 2 * P8_FBYTES,
                             a.F + ((uint64_t)(group * NV + vl) * a.m + kb * 2) * P8_FBYTES, 2 * P8_FBYTES, &full_a[s]);
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer: one M = 128, N = 64 NV MMA per 32-byte K step ----
        if (lane == 0) {
            const uint32_t id = idesc_i8(S::NPAD);
            for (uint32_t it = 0; it < nkb; it++) {
                const int sa = it % S::ASTAGES, sb = it % S::BSTAGES;
                if (!mbar_wait(&full_a[sa], (it / S::ASTAGES) & 1) || !mbar_wait(&full_b[sb], (it / S::BSTAGES) & 1)) {
                    atomicOr(a.err, 2u);
                    s_abort = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a0 = smem_u32(sA + sa * TC_A_BYTES), b0 = smem_u32(sB + sb * S::B_BYTES);
#pragma unroll
                for (int k = 0; k < 4; k++) {  // column k/2, s in [32(k%2), 32(k%2)+32): chunks 2(k%2), 2(k%2)+1
                    const uint32_t acc = (it > 0 || k > 0) ? 1u : 0u;
                    const uint32_t bcol = b0 + (k >> 1) * S::BCOL + (k & 1) * 2 * S::LBO;
                    mma_i8(tmem, sw128_desc(a0 + 32 * k), ns_desc_lbo(bcol, S::LBO), id, acc);
                }
                mma_commit(&empty_a[sa]);
                mma_commit(&empty_b[sb]);
            }
            mma_commit(done);
        }
    } else {
        // ---- B builders: thread (column jj, vector v, seq, b < 8) writes the
        // chunks c < 5 of both phases p = b + 8h (h = 0, 1), G_p = H_seq[16c + p,
        // 16c + p + 16), at [jj][c][h][seq][v][b]; the two phases share the
        // words [b/4, b/4 + 23) of the sequence, read once.  A warp covers two
        // (jj, v) pairs and both sequences, so each store phase writes whole
        // 128-byte rows and the loads touch eight distinct words ----
        const int bt = threadIdx.x - 64;
        const int b = bt & 7, seq = (bt >> 3) & 1, combo = bt >> 4;
        const int v = combo % NV, jj = combo / NV;
        const bool active = jj < 2 && (uint32_t)v < nvalid;
        for (uint32_t it = 0; it < nkb; it++) {
            const int sb = it % S::BSTAGES;
            uint32_t st = 0;  // 0 go, 1 timed out, 2 another role aborted (lane 0 waits for the warp)
            if (lane == 0) {
                const int sa = it % S::ASTAGES;
                if (!mbar_wait(&full_a[sa], (it / S::ASTAGES) & 1) ||
                    (it >= S::BSTAGES && !mbar_wait(&empty_b[sb], ((it / S::BSTAGES) & 1) ^ 1)))
                    st = 1;
                else if (s_abort)
                    st = 2;
            }
            st = __shfl_sync(0xffffffffu, st, 0);
            if (st == 1 && lane == 0) {
                atomicOr(a.err, 4u);
                s_abort = 1;
            }
            if (st) break;
            if (active) {
                const int sa = it % S::ASTAGES;
                const uint32_t* src = reinterpret_cast<const uint32_t*>(sF + sa * S::F_STAGE + (v * 2 + jj) * P8_FBYTES +
                                                                        seq * P8_HSEQ) + (b >> 2);
                uint32_t w[23];  // bytes < 96 of the 112-byte sequence
#pragma unroll
                for (int q = 0; q < 23; q++) w[q] = src[q];
                const uint32_t sh = 8 * (b & 3);
                uint8_t* dst = sB + sb * S::B_BYTES + jj * S::BCOL + seq * (NV * 128) + v * 128 + b * 16;
#pragma unroll
                for (int h = 0; h < 2; h++)
#pragma unroll
                    for (int c = 0; c < 5; c++) {
                        const int o = 4 * c + 2 * h;
                        *reinterpret_cast<uint4*>(dst + h * (2 * NV * 128) + c * S::LBO) =
                            make_uint4(__funnelshift_r(w[o], w[o + 1], sh), __funnelshift_r(w[o + 1], w[o + 2], sh),
                                       __funnelshift_r(w[o + 2], w[o + 3], sh), __funnelshift_r(w[o + 3], w[o + 4], sh));
                    }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&full_b[sb]);
        }
        // ---- epilogue (warps 2..5 cover TMEM lane groups 2, 3, 0, 1) ----
        uint32_t okw = 0;
        if (lane == 0) okw = (nkb > 0 && !s_abort && mbar_wait(done, 0)) ? 1u : 0u;
        const bool ok = __shfl_sync(0xffffffffu, okw, 0) != 0;
        if (nkb > 0 && !ok && warp < 6) atomicOr(a.err, 8u);
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int lg = warp & 3;
        const int row = lg * 32 + lane;
        int32_t* dst = a.partial + ((uint64_t)cta * 128 + row) * S::NPAD;
        for (int c0 = 0; c0 < (warp < 6 ? S::NPAD : 0); c0 += 16) {
            uint32_t v16[16];
            const uint32_t taddr = tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v16[0]), "=r"(v16[1]), "=r"(v16[2]), "=r"(v16[3]), "=r"(v16[4]), "=r"(v16[5]), "=r"(v16[6]),
                  "=r"(v16[7]), "=r"(v16[8]), "=r"(v16[9]), "=r"(v16[10]), "=r"(v16[11]), "=r"(v16[12]), "=r"(v16[13]),
                  "=r"(v16[14]), "=r"(v16[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; q += 4)
                *reinterpret_cast<int4*>(dst + c0 + q) =
                    ok ? make_int4((int)v16[q], (int)v16[q + 1], (int)v16[q + 2], (int)v16[q + 3]) : make_int4(0, 0, 0, 0);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(S::TMEM_COLS));
    }
}

// c_{v,i}[r] = sum_{ks} sum_l 2^(8l) D[ks][(i,l)][col] mod q for the column
// col of row r (no fold: the small-digit form computes mod Phi_81 directly).
// Block (group·kappa + i, y) sums the K splits [y n/S, (y+1) n/S) of row i
// (its two halves take alternate splits) into int64 slice sums; the last block
// of a row (ticket) adds the S slices and reduces mod q.  With S slices per row
// the grid fills the GPU even for a single vector (kappa rows).
template <int NV>
__global__ void __launch_bounds__(2 * P8<NV>::NPAD) commit_p8_reduce_kernel(const int32_t* __restrict__ partial,
                                                                            uint32_t n_groups, uint32_t n_ksplit,
                                                                            uint32_t kappa, uint32_t n_vec,
                                                                            int64_t* __restrict__ slices,
                                                                            uint32_t* __restrict__ tickets,
                                                                            uint64_t* __restrict__ out) {
    constexpr int NP = P8<NV>::NPAD;
    const uint32_t row = blockIdx.x, S = gridDim.y, y = blockIdx.y;
    const uint32_t group = row / kappa, i = row % kappa;
    const int col = threadIdx.x % NP, half = threadIdx.x / NP;
    __shared__ int64_t s_acc[NP][8];
    __shared__ bool s_last;
    int64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const uint32_t ks0 = (uint32_t)((uint64_t)y * n_ksplit / S), ks1 = (uint32_t)((uint64_t)(y + 1) * n_ksplit / S);
    for (uint32_t ks = ks0 + half; ks < ks1; ks += 2) {
        const int32_t* pp = partial + ((uint64_t)(ks * n_groups + group) * 128 + i * 8) * NP + col;
#pragma unroll
        for (int l = 0; l < 8; l++) acc[l] += pp[(uint64_t)l * NP];
    }
    if (half) {
#pragma unroll
        for (int l = 0; l < 8; l++) s_acc[col][l] = acc[l];
    }
    __syncthreads();
    int64_t* mine = slices + ((uint64_t)row * S + y) * 8 * NP;
    if (!half) {
#pragma unroll
        for (int l = 0; l < 8; l++) mine[l * NP + col] = acc[l] + s_acc[col][l];
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicInc(tickets + row, S - 1) == S - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // last block: half h adds the slices y = h, h + 2, ...
#pragma unroll
    for (int l = 0; l < 8; l++) acc[l] = 0;
    for (uint32_t yy = half; yy < S; yy += 2) {
        const int64_t* sl = slices + ((uint64_t)row * S + yy) * 8 * NP + col;
#pragma unroll
        for (int l = 0; l < 8; l++) acc[l] += __ldcg(sl + l * NP);
    }
    __syncthreads();
    if (half) {
#pragma unroll
        for (int l = 0; l < 8; l++) s_acc[col][l] = acc[l];
    }
    __syncthreads();
    if (half) return;
    uint64_t c = 0;
#pragma unroll
    for (int l = 0; l < 8; l++) c = gl::add(c, gl::mul(gl::from_i64(acc[l] + s_acc[col][l]), 1ULL << (8 * l)));
    const int g = col >> 3, b = col & 7;
    const int v = g % NV, seq = (g / NV) & 1, h = (g / (2 * NV)) & 1, aa = g / (4 * NV);
    const int rp = 16 * aa + 8 * h + b;
    const uint32_t vg = group * NV + v;
    if (rp >= 5 && vg < n_vec) out[((uint64_t)vg * kappa + i) * NEO_D + (seq ? 31 - rp : 58 - rp)] = c;
}

}  // namespace

// ---------------------------------------------------------------------------
int tc_pp_prepare(neo_gpu_ctx* ctx, PPEntry* pp) {
    if (pp->kappa * 8 > 128) return ctx->fail(NEO_ERR_UNSUPPORTED, "tensor-core commit: kappa <= 16");
    if (pp->m % 2) return ctx->fail(NEO_ERR_UNSUPPORTED, "tensor-core commit: m must be even");
    pp->tc = false;
    const uint64_t n_kb = pp->m / 2;
    if (!pp->d_pp_limbs) NEO_CK(ctx, cudaMalloc(&pp->d_pp_limbs, n_kb * TC_A_BYTES));  // size depends on m only
    pp_limbs_kernel<<<(unsigned)n_kb, 256, 0, ctx->stream>>>(pp->d_pp, pp->kappa, pp->m, pp->d_pp_limbs);
    NEO_LAUNCHED(ctx);
    NEO_CK(ctx, ctx_sync(ctx));
    pp->tc = true;
    return NEO_OK;
}

// Vectors per CTA: the cyclic form runs groups of 4; the small-digit form
// runs a single vector alone (the MCS commitment: N = 64, no padding
// vectors) and groups of 4 otherwise.
static uint32_t tc_nv(uint32_t n_vec, bool small) { return small && n_vec == 1 ? 1 : 4; }

// K-split slices per row of the small-digit reduce: about two blocks per SM
static uint32_t p8_slices(uint32_t n_groups, uint32_t kappa, uint32_t n_ksplit) {
    const uint32_t rows = n_groups * kappa;
    uint32_t s = (2 * 148 + rows - 1) / rows;
    return std::max(1u, std::min(s, n_ksplit));
}

size_t tc_scratch_bytes(uint32_t n_vec, uint64_t m, bool small, uint32_t kappa, uint32_t* n_groups_out,
                        uint32_t* n_ksplit_out, uint32_t* kb_per_cta_out) {
    const uint32_t nv = tc_nv(n_vec, small);
    const uint32_t n_groups = (n_vec + nv - 1) / nv;
    const uint32_t n_kb = (uint32_t)(m / 2);
    // fill whole waves of 148 SMs (1 CTA per SM), at most TC_MAX_KB K blocks per CTA
    uint32_t waves = 1, n_ksplit;
    for (;; waves++) {
        // n_groups * n_ksplit <= whole waves of 148 SMs x the CTAs one SM holds
        n_ksplit = (148 * (small && nv == 4 ? P8<4>::CTAS : 1) * waves) / n_groups;
        if (n_ksplit == 0) n_ksplit = 1;
        if (n_ksplit > n_kb) n_ksplit = n_kb;
        if ((n_kb + n_ksplit - 1) / n_ksplit <= TC_MAX_KB) break;
    }
    const uint32_t kb_per_cta = (n_kb + n_ksplit - 1) / n_ksplit;
    n_ksplit = (n_kb + kb_per_cta - 1) / kb_per_cta;
    *n_groups_out = n_groups;
    *n_ksplit_out = n_ksplit;
    *kb_per_cta_out = kb_per_cta;
    const size_t fb = small ? P8_FBYTES : TC_FBYTES, npad = small ? 64 * nv : TC_NPAD;
    size_t f_bytes = (size_t)n_vec * m * fb + 64;
    size_t p_bytes = (size_t)n_groups * n_ksplit * 128 * npad * 4;
    // small form: the reduce's int64 slice sums and one ticket per row
    size_t r_bytes = small ? (size_t)n_groups * kappa * p8_slices(n_groups, kappa, n_ksplit) * 8 * npad * 8 +
                                 (((size_t)n_groups * kappa * 4 + 255) & ~size_t(255))
                           : 0;
    return ((f_bytes + 255) & ~size_t(255)) + p_bytes + r_bytes + 256 /*flag*/ + 256;
}

template <int NV>
static int launch_p8(neo_gpu_ctx* ctx, const TcArgs& a, uint32_t kappa, uint8_t* red, uint64_t* d_out) {
    using S = P8<NV>;
    const size_t smem = S::SMEM + 1024 /*align*/ + 256 /*barriers*/;
    static SmemLimit limit;
    NEO_CK(ctx, limit.at_least(commit_p8_kernel<NV>, smem));
    const uint32_t rows = a.n_groups * kappa, ns = p8_slices(a.n_groups, kappa, a.n_ksplit);
    int64_t* slices = reinterpret_cast<int64_t*>(red);
    uint32_t* tickets = reinterpret_cast<uint32_t*>(red + (size_t)rows * ns * 8 * S::NPAD * 8);
    NEO_CK(ctx, cudaMemsetAsync(tickets, 0, (size_t)rows * 4, ctx->stream));
    commit_p8_kernel<NV><<<a.n_groups * a.n_ksplit, S::THREADS, smem, ctx->stream>>>(a);
    NEO_LAUNCHED(ctx);
    commit_p8_reduce_kernel<NV><<<dim3(rows, ns), 2 * S::NPAD, 0, ctx->stream>>>(
        a.partial, a.n_groups, a.n_ksplit, kappa, a.n_vec, slices, tickets, d_out);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}

int launch_commit_tc(neo_gpu_ctx* ctx, const PPEntry* pp, const int8_t* d_digits, uint32_t n_vec, uint64_t* d_out,
                     uint8_t* scratch, uint32_t* d_err, int digits) {
    const uint64_t m = pp->m;
    TcArgs a;
    a.ppl = pp->d_pp_limbs;
    a.err = d_err;
    a.m = m;
    a.n_vec = n_vec;
    a.n_kb = (uint32_t)(m / 2);
    if (digits != TC_DIGITS_ANY) {
        // small-digit form; for digits of unknown size the window sequences are
        // built first and checked (one synchronisation), falling back to the
        // cyclic form when an entry leaves int8
        uint32_t n_groups, n_ksplit, kb_per_cta;
        const size_t need = tc_scratch_bytes(n_vec, m, true, pp->kappa, &n_groups, &n_ksplit, &kb_per_cta);
        uint8_t* F = scratch;
        const size_t f_end = ((size_t)n_vec * m * P8_FBYTES + 64 + 255) & ~size_t(255);
        uint32_t* flag = reinterpret_cast<uint32_t*>(scratch + need - 512);
        const bool known = digits == TC_DIGITS_SMALL;
        if (!known) NEO_CK(ctx, cudaMemsetAsync(flag, 0, 4, ctx->stream));
        p8_seq_kernel<<<ceil_div((uint64_t)n_vec * m, P8_SEQ_THREADS), P8_SEQ_THREADS, 0, ctx->stream>>>(
            d_digits, n_vec, m, F, known ? d_err : flag);
        NEO_LAUNCHED(ctx);
        bool ok = true;
        if (!known) {
            uint32_t h_flag = 0;
            NEO_CK(ctx, ctx_d2h(ctx, &h_flag, flag, 4));
            NEO_CK(ctx, ctx_sync(ctx));
            ok = h_flag == 0;
        }
        if (ok) {
            a.F = F;
            a.partial = reinterpret_cast<int32_t*>(scratch + f_end);
            a.n_groups = n_groups;
            a.n_ksplit = n_ksplit;
            a.kb_per_cta = kb_per_cta;
            uint8_t* red = scratch + f_end + (size_t)n_groups * n_ksplit * 128 * 64 * tc_nv(n_vec, true) * 4;
            return tc_nv(n_vec, true) == 1 ? launch_p8<1>(ctx, a, pp->kappa, red, d_out)
                                           : launch_p8<4>(ctx, a, pp->kappa, red, d_out);
        }
    }
    uint32_t n_groups, n_ksplit, kb_per_cta;
    tc_scratch_bytes(n_vec, m, false, pp->kappa, &n_groups, &n_ksplit, &kb_per_cta);
    uint8_t* F = scratch;
    int32_t* partial = reinterpret_cast<int32_t*>(scratch + (((size_t)n_vec * m * TC_FBYTES + 64 + 255) & ~size_t(255)));
    f_seq_kernel<<<ceil_div((uint64_t)n_vec * m, 128), 128, 0, ctx->stream>>>(d_digits, n_vec, m, F);
    NEO_LAUNCHED(ctx);
    a.F = F;
    a.partial = partial;
    a.n_groups = n_groups;
    a.n_ksplit = n_ksplit;
    a.kb_per_cta = kb_per_cta;
    const size_t smem = TC_SMEM_BYTES + 1024 /*align*/ + 256 /*barriers*/;
    static SmemLimit limit;
    NEO_CK(ctx, limit.at_least(commit_tc_kernel, smem));
    commit_tc_kernel<<<n_groups * n_ksplit, TC_THREADS, smem, ctx->stream>>>(a);
    NEO_LAUNCHED(ctx);
    commit_tc_reduce_kernel<<<n_groups * pp->kappa, RED_THREADS, 0, ctx->stream>>>(partial, n_groups, n_ksplit,
                                                                                     pp->kappa, n_vec, d_out);
    NEO_LAUNCHED(ctx);
    return NEO_OK;
}
