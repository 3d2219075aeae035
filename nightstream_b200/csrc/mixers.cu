// mixers.cu -- the commitment mixers of the shard loop (CommitMixers,
// crates/neo-fold/src/shard.rs:146-153) as C-ABI calls:
//   mix_rhos_commits(rho, cs) = sum_i rho_i c_i   (S-action of 54 x 54 F_q
//                                                  matrices on commitments)
//   combine_b_pows(cs, b)     = sum_i b^i c_i      (the DEC parent check)
// Commitments are kappa columns of 54 F_q (Commitment::data column-major,
// crates/neo-ajtai/src/types.rs:15-22).  The fold step mixes its own
// commitments on the device (rot_mix_kernel in fold.cu, small-integer rho);
// these entry points take general matrices so a caller's CommitMixers
// closures can drop onto the GPU unchanged.
#include "internal.cuh"

using gl::K;

namespace {

// out[c][r] = sum_i sum_k rho_i[r][k] cs_i[c][k]; one thread per (c, r), the
// count * 54 products summed unreduced and reduced once.
__global__ void __launch_bounds__(64) mix_rhos_kernel(const uint64_t* __restrict__ rhos,
                                                      const uint64_t* __restrict__ cs, uint32_t count,
                                                      uint32_t kappa, uint64_t* __restrict__ out) {
    const uint32_t c = blockIdx.x, r = threadIdx.x;
    if (r >= NEO_D) return;
    gl::Acc160 acc;
    gl::acc_zero(acc);
    for (uint32_t i = 0; i < count; i++) {
        const uint64_t* R = rhos + ((uint64_t)i * NEO_D + r) * NEO_D;
        const uint64_t* C = cs + ((uint64_t)i * kappa + c) * NEO_D;
        for (int k = 0; k < NEO_D; k++) gl::acc_mad(acc, R[k], C[k]);
    }
    out[(uint64_t)c * NEO_D + r] = gl::acc_reduce(acc);
}

// out[c][r] = sum_i b^i cs_i[c][r]
__global__ void combine_b_pows_kernel(const uint64_t* __restrict__ cs, uint32_t count, uint32_t len, uint64_t b,
                                      uint64_t* __restrict__ out) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= len) return;
    gl::Acc160 acc;
    gl::acc_zero(acc);
    uint64_t pw = 1;
    for (uint32_t i = 0; i < count; i++) {
        gl::acc_mad(acc, pw, cs[(uint64_t)i * len + e]);
        pw = gl::mul(pw, b);
    }
    out[e] = gl::acc_reduce(acc);
}

}  // namespace

static int neo_gpu_mix_rhos_commits_impl_abi(neo_gpu_ctx* ctx, const uint64_t* rhos, const uint64_t* cs,
                                             uint32_t count, uint32_t kappa, uint64_t* out) {
    if (!ctx) return NEO_ERR_ARG;
    if (!rhos || !cs || !out || count == 0 || kappa == 0 || count > (1u << 20))
        return ctx->fail(NEO_ERR_ARG, "mix_rhos_commits: bad args");
    NEO_CK(ctx, cudaSetDevice(ctx->device));
    DevBuf<uint64_t> dr, dc, dout;
    NEO_CK(ctx, dr.alloc((size_t)count * NEO_D * NEO_D));
    NEO_CK(ctx, dc.alloc((size_t)count * kappa * NEO_D));
    NEO_CK(ctx, dout.alloc((size_t)kappa * NEO_D));
    NEO_CK(ctx, cudaMemcpyAsync(dr.p, rhos, dr.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    NEO_CK(ctx, cudaMemcpyAsync(dc.p, cs, dc.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    mix_rhos_kernel<<<kappa, 64, 0, ctx->stream>>>(dr.p, dc.p, count, kappa, dout.p);
    NEO_LAUNCHED(ctx);
    NEO_CK(ctx, ctx_d2h(ctx, out, dout.p, dout.bytes()));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_mix_rhos_commits(neo_gpu_ctx* ctx, const uint64_t* rhos, const uint64_t* cs, uint32_t count,
                                        uint32_t kappa, uint64_t* out) {
    NEO_ABI_GUARD(neo_gpu_mix_rhos_commits_impl_abi(ctx, rhos, cs, count, kappa, out))
}

static int neo_gpu_combine_b_pows_impl_abi(neo_gpu_ctx* ctx, const uint64_t* cs, uint32_t count, uint32_t kappa,
                                           uint32_t b, uint64_t* out) {
    if (!ctx) return NEO_ERR_ARG;
    if (!cs || !out || count == 0 || kappa == 0 || count > (1u << 20))
        return ctx->fail(NEO_ERR_ARG, "combine_b_pows: bad args");
    NEO_CK(ctx, cudaSetDevice(ctx->device));
    const uint32_t len = kappa * NEO_D;
    DevBuf<uint64_t> dc, dout;
    NEO_CK(ctx, dc.alloc((size_t)count * len));
    NEO_CK(ctx, dout.alloc(len));
    NEO_CK(ctx, cudaMemcpyAsync(dc.p, cs, dc.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    combine_b_pows_kernel<<<ceil_div(len, 128), 128, 0, ctx->stream>>>(dc.p, count, len, gl::canon(b), dout.p);
    NEO_LAUNCHED(ctx);
    NEO_CK(ctx, ctx_d2h(ctx, out, dout.p, dout.bytes()));
    NEO_CK(ctx, ctx_sync(ctx));
    return NEO_OK;
}
extern "C" int neo_gpu_combine_b_pows(neo_gpu_ctx* ctx, const uint64_t* cs, uint32_t count, uint32_t kappa, uint32_t b,
                                      uint64_t* out) {
    NEO_ABI_GUARD(neo_gpu_combine_b_pows_impl_abi(ctx, cs, count, kappa, b, out))
}
