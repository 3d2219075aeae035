// fold.cu -- device-resident Neo fold step for one shard (main lane, no
// Twist/Shout): MCS commit -> Pi_CCS (batched time rounds + Ajtai rounds) ->
// ME outputs -> Pi_RLC -> Pi_DEC (12 child commitments + child ME claims).
//
// Reference: fold_shard_prove_impl (crates/neo-fold/src/shard.rs:1725-2283),
// prove_rlc_dec_lane (shard.rs:1170-1331), prove_route_a_batched_time
// (crates/neo-fold/src/memory_sidecar/route_a_time.rs:28-152), the sum-check
// drivers (crates/neo-reductions/src/sumcheck.rs:124-456) and their domain
// separation (memory_sidecar/sumcheck_ds.rs:11-77).  The transcript calls are
// issued in the reference's order with the reference's labels.
//
// All witness digit planes live in one device buffer Zall[1 + k_rho][54][m]:
// slot 0 holds the step's MCS witness, slots 1..k_rho the carried children.
// Pi_DEC writes the new children straight into slots 1..k_rho.
#include "internal.cuh"
#include "transcript.h"
#include <algorithm>
#include <chrono>
#include <memory>

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
    std::vector<K> y;             // t * 2^ell_d (padded)
    std::vector<K> ysc;           // t
    uint32_t m_in = 0;
    uint8_t digest[32] = {0};
};

static std::vector<uint8_t> le64(uint64_t v) {
    std::vector<uint8_t> b(8);
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * i));
    return b;
}

// out[v][r] = sum_i rot_i[r][k] * V_i[v][k]  over F_q, element stride `stride`
// (Commitment mixing mix_rhos_commits and S-action on y vectors, common.rs:398-430).
__global__ void rot_mix_kernel(const int8_t* __restrict__ rot, uint32_t count, const uint64_t* __restrict__ V,
                               uint32_t nv, uint32_t stride, uint64_t* __restrict__ out) {
    const uint32_t v = blockIdx.x / stride, comp = blockIdx.x % stride;
    const int r = threadIdx.x;
    if (r >= NEO_D) return;
    uint64_t acc = 0;
    for (uint32_t i = 0; i < count; i++) {
        const int8_t* R = rot + (size_t)i * NEO_D * NEO_D + r * NEO_D;
        const uint64_t* x = V + (((size_t)i * nv + v) * NEO_D) * stride + comp;
        for (int k = 0; k < NEO_D; k++) {
            int c = R[k];
            if (c == 0) continue;
            uint64_t xv = x[(size_t)k * stride];
            uint64_t p = c > 0 ? gl::mul_small(xv, (uint32_t)c) : gl::neg(gl::mul_small(xv, (uint32_t)(-c)));
            acc = gl::add(acc, p);
        }
    }
    out[((size_t)v * NEO_D + r) * stride + comp] = acc;
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

}  // namespace

// ---------------------------------------------------------------------------
struct neo_gpu_shard {
    neo_gpu_ctx* ctx = nullptr;
    DevCcs ccs;
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
};

using hclock = std::chrono::steady_clock;
static inline double ms_since(hclock::time_point t0) {
    return std::chrono::duration<double, std::milli>(hclock::now() - t0).count();
}

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
static void ccs_digest_words(const neo_ccs_desc* d, uint64_t* out4) {
    const neo::Poseidon2W16& P = neo::digest_perm();
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
            // row-major enumeration, columns ascending within a row
            const uint64_t* cp = d->col_ptr + (size_t)j * (d->m + 1);
            uint64_t base = d->nnz_off[j], nnz = d->nnz_off[j + 1] - base;
            std::vector<uint64_t> off(d->n + 1, 0);
            for (uint64_t k = 0; k < nnz; k++) off[d->row_idx[base + k] + 1]++;
            for (uint32_t r = 0; r < d->n; r++) off[r + 1] += off[r];
            std::vector<std::pair<uint64_t, uint64_t>> ent(nnz);
            std::vector<uint64_t> wp(off.begin(), off.end() - 1);
            for (uint32_t c = 0; c < d->m; c++)
                for (uint64_t k = cp[c]; k < cp[c + 1]; k++) ent[wp[d->row_idx[base + k]]++] = {c, d->vals[base + k]};
            for (uint32_t r = 0; r < d->n; r++)
                for (uint64_t e = off[r]; e < off[r + 1]; e++) emit(r, ent[e].first, ent[e].second);
        }
        P.permute(st);
    }
    for (int i = 0; i < 4; i++) out4[i] = st[i];
}

extern "C" int neo_ccs_digest(const neo_ccs_desc* d, uint64_t* out4) {
    if (!d || !out4 || d->t == 0 || d->n == 0 || d->m == 0) return NEO_ERR_ARG;
    ccs_digest_words(d, out4);
    return NEO_OK;
}

extern "C" int neo_gpu_shard_create(neo_gpu_ctx* ctx, const neo_ccs_desc* desc, uint32_t m_in, uint32_t k_rho,
                                    const char* app_label, neo_gpu_shard** out) {
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
    NEO_CK(ctx, sh->Zall.alloc((size_t)(1 + k_rho) * NEO_D * m));
    NEO_CK(ctx, sh->d_z.alloc(m));
    NEO_CK(ctx, sh->d_mix.alloc((size_t)NEO_D * m));
    NEO_CK(ctx, sh->d_rot.alloc((size_t)(1 + k_rho) * NEO_D * NEO_D));
    NEO_CK(ctx, sh->d_commits.alloc((size_t)(1 + k_rho) * sh->kappa * NEO_D));
    NEO_CK(ctx, sh->d_flags.alloc(2));
    NEO_CK(ctx, sh->d_ychild.alloc((size_t)k_rho * sh->t * NEO_D));
    size_t mixv = (size_t)(1 + k_rho) * std::max<uint32_t>(sh->kappa, 2 * sh->t + m_in) * NEO_D * 2;
    NEO_CK(ctx, sh->d_mixv.alloc(mixv));
    NEO_CK(ctx, sh->d_mixo.alloc(mixv));
    *out = guard.release();
    return NEO_OK;
}

extern "C" int neo_gpu_shard_destroy(neo_gpu_shard* sh) {
    if (!sh) return NEO_ERR_ARG;
    cudaSetDevice(sh->ctx->device);
    cudaStreamSynchronize(sh->ctx->stream);
    if (sh->orc) neo_gpu_ccs_oracle_destroy(sh->orc);
    delete sh;
    return NEO_OK;
}

// ---------------------------------------------------------------------------
// one fold step
// ---------------------------------------------------------------------------
namespace {

struct Rounds {
    std::vector<K> coeffs;  // rounds x (d_sc+1)
    std::vector<K> chals;
};

static void interpolate(const std::vector<K>& xs, const std::vector<K>& ys, std::vector<K>& co) {
    // sumcheck.rs:74-118
    const size_t n = xs.size();
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
        K den = gl::kone();
        for (size_t j = 0; j < n; j++)
            if (i != j) den = gl::kmul(den, gl::ksub(xs[i], xs[j]));
        K sc = gl::kmul(ys[i], gl::kinv(den));
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

}  // namespace

int ccs_oracle_create_dev(neo_gpu_ctx* ctx, const DevCcs* ccs, const int8_t* d_Z, uint32_t k, uint32_t b,
                          const K* alpha, const K* beta_a, const K* beta_r, K gamma, const K* r_inputs,
                          uint32_t ell_d, uint32_t ell_n, uint32_t d_sc, neo_gpu_ccs_oracle** out);
int ccs_oracle_dev_vj(neo_gpu_ccs_oracle* o, const K** vj);

static int fold_step_impl(neo_gpu_shard* sh, const uint64_t* z_host, const uint64_t* d_z_in) {
    neo_gpu_ctx* ctx = sh->ctx;
    neo::Transcript& tr = *sh->tr;
    const uint64_t m = sh->m;
    const uint32_t kappa = sh->kappa, t = sh->t, ell_n = sh->ell_n, ell_d = sh->ell_d, d_sc = sh->d_sc;
    const uint32_t idx = sh->step_idx;
    const uint32_t n_acc = (uint32_t)sh->acc.size();
    const uint32_t k = 1 + n_acc;
    const uint32_t d_pad = 1u << ell_d;
    std::vector<uint64_t>& P = sh->proof;
    P.clear();
    int rc;
    const auto t_step = hclock::now();
    const uint64_t perms0 = tr.permutations();
    for (double& v : sh->stats) v = 0;
    auto t_ph = hclock::now();

    // ---- witness build: z -> Z (decomp) -> c = commit(Z)  (session.rs:977-978) ----
    const uint64_t* d_z = d_z_in;
    if (z_host) {
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_z.p, z_host, m * 8, cudaMemcpyHostToDevice, ctx->stream));
        d_z = sh->d_z.p;
    }
    decomp_b2_kernel<<<ceil_div(m, 256), 256, 0, ctx->stream>>>(d_z, m, sh->Zall.p);
    NEO_LAUNCHED(ctx);
    if ((rc = launch_commit(ctx, sh->Zall.p, 1, m, sh->d_commits.p))) return rc;
    MeInst mcs;
    mcs.c.resize((size_t)kappa * NEO_D);
    std::vector<uint64_t> x(sh->m_in);
    std::vector<int8_t> Xd((size_t)NEO_D * sh->m_in);
    NEO_CK(ctx, cudaMemcpyAsync(mcs.c.data(), sh->d_commits.p, mcs.c.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(x.data(), d_z, sh->m_in * 8, cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, cudaMemcpy2DAsync(Xd.data(), sh->m_in, sh->Zall.p, m, sh->m_in, NEO_D, cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, cudaStreamSynchronize(ctx->stream));
    if ((rc = check_device_error(ctx))) return rc;
    for (auto& v : x) v = gl::canon(v);
    mcs.m_in = sh->m_in;
    mcs.X.resize(Xd.size());
    for (size_t i = 0; i < Xd.size(); i++) mcs.X[i] = gl::from_i64(Xd[i]);
    P.insert(P.end(), mcs.c.begin(), mcs.c.end());
    sh->stats[1] = ms_since(t_ph);
    t_ph = hclock::now();

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
    // ---- claimed_initial_sum_from_inputs (optimized_engine/common.rs:839-947) ----
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
    P.push_back(T.re);
    P.push_back(T.im);
    // ---- r_cycle = sample_ext_point (neo-memory/src/ts_common.rs:22-37) ----
    for (uint32_t i = 0; i < ell_n; i++) {
        auto b8 = le64(i);
        tr.append_message("route_a/r_cycle", b8.data(), 8);
        tr.challenge_field("route_a/cycle/0");
        tr.challenge_field("route_a/cycle/1");
    }

    sh->stats[2] = ms_since(t_ph);
    t_ph = hclock::now();
    // ---- Pi_CCS oracle over Zall slots 0..n_acc (workspace reused across steps) ----
    const K* rin = n_acc ? sh->acc[0].r.data() : nullptr;
    if ((rc = ccs_oracle_create_dev(ctx, &sh->ccs, sh->Zall.p, k, sh->b, alpha.data(), beta_a.data(), beta_r.data(),
                                    gamma, rin, ell_d, ell_n, d_sc, &sh->orc)))
        return rc;
    neo_gpu_ccs_oracle* orc = sh->orc;

    sh->stats[3] = ms_since(t_ph);
    t_ph = hclock::now();
    std::vector<K> xs(d_sc + 1), ys(d_sc + 1), co;
    for (uint32_t i = 0; i <= d_sc; i++) xs[i] = gl::kfq(i);
    // ---- batched time sum-check, one claim "ccs/time" (route_a_time.rs:28-152) ----
    {
        auto b1 = le64(1), b0 = le64(0), bd = le64(d_sc);
        tr.append_message("batched/dynamic_bind/len", b1.data(), 8);
        tr.append_message("batched/dynamic_bind/claim_label", "ccs/time");
        tr.append_message("batched/dynamic_bind/claim_idx", b0.data(), 8);
        tr.append_message("batched/dynamic_bind/degree_bound", bd.data(), 8);
        uint8_t one = 1;
        tr.append_message("batched/dynamic_bind/is_dynamic", &one, 1);
        absorb_k(tr, "batched/dynamic_bind/claimed_sum", T);
    }
    auto bidx = le64(idx);
    tr.append_message("sc/domain", "shard/batched_time");
    tr.append_message("sc/inst_idx", bidx.data(), 8);
    K running = T;
    std::vector<K> r_time;
    for (uint32_t rd = 0; rd < ell_n; rd++) {
        auto br = le64(rd);
        tr.append_message("batched/round_idx", br.data(), 8);
        if ((rc = neo_gpu_ccs_oracle_evals(orc, (const uint64_t*)xs.data(), d_sc + 1, (uint64_t*)ys.data()))) return rc;
        K s01 = gl::kadd(ys[0], ys[1]);
        if (s01.re != running.re || s01.im != running.im)
            return ctx->fail(NEO_ERR_INVARIANT, "batched sum-check: p(0)+p(1) != running sum");
        interpolate(xs, ys, co);
        tr.append_message("batched/claim_label", "ccs/time");
        auto b0 = le64(0);
        tr.append_message("batched/claim_idx", b0.data(), 8);
        for (auto& c : co) absorb_k(tr, "batched/round/coeff", c);
        uint64_t c0 = tr.challenge_field("batched/challenge/0");
        uint64_t c1 = tr.challenge_field("batched/challenge/1");
        K r = gl::kmk(c0, c1);
        r_time.push_back(r);
        running = poly_eval(co, r);
        if ((rc = neo_gpu_ccs_oracle_fold(orc, (const uint64_t*)&r))) return rc;
        for (auto& c : co) { P.push_back(c.re); P.push_back(c.im); }
    }
    tr.append_message("sc/domain_end", "shard/batched_time");
    tr.append_message("sc/inst_idx_end", bidx.data(), 8);
    sh->stats[4] = ms_since(t_ph);
    t_ph = hclock::now();
    // ---- Ajtai rounds: run_sumcheck_prover_ds("ccs/ajtai") ----
    tr.append_message("sc/domain", "ccs/ajtai");
    tr.append_message("sc/inst_idx", bidx.data(), 8);
    absorb_k(tr, "sc/claimed_sum", running);
    for (uint32_t rd = 0; rd < ell_d; rd++) {
        if ((rc = neo_gpu_ccs_oracle_evals(orc, (const uint64_t*)xs.data(), d_sc + 1, (uint64_t*)ys.data()))) return rc;
        K s01 = gl::kadd(ys[0], ys[1]);
        if (s01.re != running.re || s01.im != running.im)
            return ctx->fail(NEO_ERR_INVARIANT, "Ajtai sum-check: p(0)+p(1) != running sum");
        interpolate(xs, ys, co);
        for (auto& c : co) absorb_k(tr, "sumcheck/round/coeff", c);
        uint64_t c0 = tr.challenge_field("sumcheck/challenge/0");
        uint64_t c1 = tr.challenge_field("sumcheck/challenge/1");
        K r = gl::kmk(c0, c1);
        running = poly_eval(co, r);
        if ((rc = neo_gpu_ccs_oracle_fold(orc, (const uint64_t*)&r))) return rc;
        for (auto& c : co) { P.push_back(c.re); P.push_back(c.im); }
    }
    tr.append_message("sc/domain_end", "ccs/ajtai");
    tr.append_message("sc/inst_idx_end", bidx.data(), 8);
    P.push_back(running.re);
    P.push_back(running.im);
    uint8_t fold_digest[32];
    tr.digest32(fold_digest);

    sh->stats[5] = ms_since(t_ph);
    t_ph = hclock::now();
    // ---- ME outputs (oracle.rs:1955-2072) ----
    std::vector<K> y_eval((size_t)k * t * NEO_D), y_sc((size_t)k * t);
    if ((rc = neo_gpu_ccs_oracle_me_outputs(orc, (uint64_t*)y_eval.data(), (uint64_t*)y_sc.data()))) return rc;
    std::vector<MeInst> outs(k);
    for (uint32_t i = 0; i < k; i++) {
        MeInst& o = outs[i];
        const MeInst& src = i == 0 ? mcs : sh->acc[i - 1];
        o.c = src.c;
        o.X = src.X;
        o.m_in = src.m_in;
        o.r = r_time;
        o.y.assign((size_t)t * d_pad, gl::kzero());
        for (uint32_t j = 0; j < t; j++)
            for (int rho = 0; rho < NEO_D; rho++) o.y[j * d_pad + rho] = y_eval[((size_t)i * t + j) * NEO_D + rho];
        o.ysc.assign(y_sc.begin() + (size_t)i * t, y_sc.begin() + (size_t)(i + 1) * t);
        memcpy(o.digest, fold_digest, 32);
    }
    for (auto& v : y_eval) { P.push_back(v.re); P.push_back(v.im); }
    for (auto& v : y_sc) { P.push_back(v.re); P.push_back(v.im); }

    sh->stats[6] = ms_since(t_ph);
    t_ph = hclock::now();
    // ---- Pi_RLC: bind_rlc_inputs (shard.rs:1125-1168) + sample_rot_rhos_n (common.rs:467-573) ----
    tr.append_message("fold/rlc_inputs/v1", "main");
    uint64_t si = idx, mc = k;
    tr.append_u64s("step_idx", &si, 1);
    tr.append_u64s("me_count", &mc, 1);
    for (auto& me : outs) {
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
    std::vector<int8_t> rhos((size_t)k * NEO_D);
    static const int8_t A5[5] = {-2, -1, 0, 1, 2};
    for (uint32_t i = 0; i < k; i++) {
        auto bi = le64(i);
        tr.append_message("rlc/rot/index", bi.data(), 8);
        // draw_alphabet_vector (common.rs:432-465): 16-bit chunks of digest32, rejection >= 65535
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
    if ((rc = rlc_mix_device(ctx, rhos.data(), sh->Zall.p, k, m, sh->d_mix.p, sh->d_rot.p))) return rc;
    // parent commitment and y: rot mixes of the k commitments / y vectors
    {
        std::vector<uint64_t> cv((size_t)k * kappa * NEO_D);
        for (uint32_t i = 0; i < k; i++) memcpy(&cv[(size_t)i * kappa * NEO_D], outs[i].c.data(), kappa * NEO_D * 8);
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_mixv.p, cv.data(), cv.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
        rot_mix_kernel<<<kappa, 64, 0, ctx->stream>>>(sh->d_rot.p, k, sh->d_mixv.p, kappa, 1, sh->d_mixo.p);
        NEO_LAUNCHED(ctx);
    }
    std::vector<uint64_t> c_parent((size_t)kappa * NEO_D);
    NEO_CK(ctx, cudaMemcpyAsync(c_parent.data(), sh->d_mixo.p, c_parent.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<K> y_parent((size_t)t * NEO_D);
    {
        // y vectors as [k][t][54] K = stride-2 F_q
        NEO_CK(ctx, cudaMemcpyAsync(sh->d_mixv.p, y_eval.data(), y_eval.size() * 16, cudaMemcpyHostToDevice, ctx->stream));
        rot_mix_kernel<<<t * 2, 64, 0, ctx->stream>>>(sh->d_rot.p, k, sh->d_mixv.p, t, 2, sh->d_mixo.p);
        NEO_LAUNCHED(ctx);
        NEO_CK(ctx, cudaMemcpyAsync(y_parent.data(), sh->d_mixo.p, y_parent.size() * 16, cudaMemcpyDeviceToHost, ctx->stream));
    }
    P.insert(P.end(), c_parent.begin(), c_parent.end());

    sh->stats[7] = ms_since(t_ph);
    t_ph = hclock::now();
    // ---- Pi_DEC: split into k_rho planes (slots 1..k_rho), commit, child claims ----
    int8_t* planes = sh->Zall.p + (size_t)NEO_D * m;
    if ((rc = split_b_device(ctx, sh->d_mix.p, (uint64_t)NEO_D * m, sh->k_rho, sh->b, planes, sh->d_flags.p))) return rc;
    if ((rc = launch_commit(ctx, planes, sh->k_rho, m, sh->d_commits.p))) return rc;
    const K* vj = nullptr;
    if ((rc = ccs_oracle_dev_vj(orc, &vj))) return rc;
    child_y_kernel<<<sh->k_rho * NEO_D, 256, 0, ctx->stream>>>(planes, m, t, vj, sh->d_ychild.p);
    NEO_LAUNCHED(ctx);
    uint32_t flags[2];
    std::vector<uint64_t> cc((size_t)sh->k_rho * kappa * NEO_D);
    std::vector<K> yc((size_t)sh->k_rho * t * NEO_D);
    std::vector<int8_t> Xc((size_t)sh->k_rho * NEO_D * sh->m_in);
    NEO_CK(ctx, cudaMemcpyAsync(flags, sh->d_flags.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(cc.data(), sh->d_commits.p, cc.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(yc.data(), sh->d_ychild.p, yc.size() * 16, cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, cudaMemcpy2DAsync(Xc.data(), sh->m_in, planes, m, sh->m_in, (size_t)sh->k_rho * NEO_D,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    NEO_CK(ctx, cudaStreamSynchronize(ctx->stream));
    if ((rc = check_device_error(ctx))) return rc;
    if (flags[0]) return ctx->fail(NEO_ERR_INVARIANT, "DEC split: Z_mix entry out of range for k_rho digits");
    // DEC public checks (dec_children_with_commit_cached): c and y recompose in base b
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
            if (ysum[q].re != y_parent[q].re || ysum[q].im != y_parent[q].im)
                return ctx->fail(NEO_ERR_INVARIANT, "DEC public check failed (y)");
    }
    // new accumulator = children
    std::vector<MeInst> children(sh->k_rho);
    uint64_t pwb[NEO_D];
    pwb[0] = 1;
    for (int q = 1; q < NEO_D; q++) pwb[q] = gl::mul(pwb[q - 1], sh->b);
    for (uint32_t i = 0; i < sh->k_rho; i++) {
        MeInst& ch = children[i];
        ch.c.assign(cc.begin() + (size_t)i * kappa * NEO_D, cc.begin() + (size_t)(i + 1) * kappa * NEO_D);
        ch.X.resize((size_t)NEO_D * sh->m_in);
        for (size_t q = 0; q < ch.X.size(); q++) ch.X[q] = gl::from_i64(Xc[(size_t)i * NEO_D * sh->m_in + q]);
        ch.r = r_time;
        ch.m_in = sh->m_in;
        ch.y.assign((size_t)t * d_pad, gl::kzero());
        ch.ysc.resize(t);
        for (uint32_t j = 0; j < t; j++) {
            K s = gl::kzero();
            for (int rho = 0; rho < NEO_D; rho++) {
                K v = yc[((size_t)i * t + j) * NEO_D + rho];
                ch.y[j * d_pad + rho] = v;
                s = gl::kadd(s, gl::kscale(v, pwb[rho]));
            }
            ch.ysc[j] = s;
        }
        memcpy(ch.digest, fold_digest, 32);
        P.insert(P.end(), ch.c.begin(), ch.c.end());
        for (uint32_t j = 0; j < t; j++)
            for (int rho = 0; rho < NEO_D; rho++) { P.push_back(ch.y[j * d_pad + rho].re); P.push_back(ch.y[j * d_pad + rho].im); }
    }
    sh->acc.swap(children);
    sh->step_idx++;
    sh->stats[8] = ms_since(t_ph);
    sh->stats[0] = ms_since(t_step);
    sh->stats[9] = (double)(tr.permutations() - perms0);
    return NEO_OK;
}

extern "C" int neo_gpu_shard_fold_step(neo_gpu_shard* sh, const uint64_t* z, uint64_t* proof, uint64_t proof_cap,
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

// Variant with the step witness already resident on the device (d_z: m words).
extern "C" int neo_gpu_shard_fold_step_device(neo_gpu_shard* sh, const uint64_t* d_z, uint64_t* proof_len) {
    if (!sh) return NEO_ERR_ARG;
    if (!d_z) return sh->ctx->fail(NEO_ERR_ARG, "fold_step_device: null witness");
    cudaSetDevice(sh->ctx->device);
    int rc = fold_step_impl(sh, nullptr, d_z);
    if (rc) return rc;
    if (proof_len) *proof_len = sh->proof.size();
    return NEO_OK;
}

extern "C" int neo_gpu_shard_transcript_state(const neo_gpu_shard* sh, uint64_t* st8) {
    if (!sh || !st8) return NEO_ERR_ARG;
    memcpy(st8, sh->tr->state(), 64);
    return NEO_OK;
}

extern "C" int neo_gpu_shard_ccs_digest(const neo_gpu_shard* sh, uint64_t* d4) {
    if (!sh || !d4) return NEO_ERR_ARG;
    memcpy(d4, sh->mat_digest, 32);
    return NEO_OK;
}

extern "C" int neo_gpu_shard_step_stats(const neo_gpu_shard* sh, double* out, uint32_t n) {
    if (!sh || !out) return NEO_ERR_ARG;
    for (uint32_t i = 0; i < n && i < 12; i++) out[i] = sh->stats[i];
    return NEO_OK;
}
