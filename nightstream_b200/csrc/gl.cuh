// gl.cuh -- Goldilocks F_q and K = F_q[u]/(u^2 - 7) arithmetic for sm_100a.
//
// q = 2^64 - 2^32 + 1 (crates/neo-math/src/field.rs:10-16).  Elements are
// canonical u64 < q.  Products use mul.lo/mul.hi (64x64 -> 128) and the
// reduction 2^64 = 2^32 - 1, 2^96 = -1 (mod q).  K elements are (re, im) with
// u^2 = 7 (crates/neo-math/src/s_action.rs:65).
#pragma once
#include <cstdint>

#define GL_Q 0xFFFFFFFF00000001ULL
#define GL_EPS 0xFFFFFFFFULL

#ifdef __CUDACC__
#define GL_HD __host__ __device__ __forceinline__
#else
#define GL_HD inline
#endif

namespace gl {

// Branch-free forms: field elements are data-dependent, so conditional
// corrections are written as masks (no mispredicted branches on the host,
// predicated selects on the device).
GL_HD uint64_t canon(uint64_t a) { return a - ((uint64_t)(a >= GL_Q) * GL_Q); }

GL_HD uint64_t add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    s += (uint64_t)(s < a) * GL_EPS;  // carry: 2^64 = 2^32 - 1 (mod q)
    return canon(s);
}

GL_HD uint64_t sub(uint64_t a, uint64_t b) {
    uint64_t d = a - b;
    return d + (uint64_t)(a < b) * GL_Q;  // a - b + q, exact mod 2^64
}

GL_HD uint64_t neg(uint64_t a) { return a ? GL_Q - a : 0ULL; }

GL_HD uint64_t reduce128(uint64_t lo, uint64_t hi) {
    uint64_t hi_hi = hi >> 32;
    uint64_t hi_lo = hi & GL_EPS;
    uint64_t t0 = lo - hi_hi;
    t0 -= (uint64_t)(lo < hi_hi) * GL_EPS;  // borrow: -2^64 = -(2^32 - 1)
    uint64_t t1 = (hi_lo << 32) - hi_lo;     // hi_lo * (2^32 - 1)
    uint64_t s = t0 + t1;
    s += (uint64_t)(s < t0) * GL_EPS;       // carry
    return canon(s);
}

GL_HD uint64_t mulhi(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

#ifdef __CUDA_ARCH__
// a b (mod q) on the device: the four 32 x 32 partial products of a b in one
// carry chain (the two 64-bit halves of the product computed separately
// would repeat the cross terms), then reduce128 on the limbs
// (lo, r2 + 2^32 r3) with lo = r0 + 2^32 r1.
__device__ __forceinline__ uint64_t mul_dev(uint64_t a, uint64_t b) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint32_t r0, r1, r2, r3;
    asm("{\n\t"
        "mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "addc.u32 %3, 0, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, %3;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
    return reduce128(((uint64_t)r1 << 32) | r0, ((uint64_t)r3 << 32) | r2);
}
#endif

GL_HD uint64_t mul(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return mul_dev(a, b);
#else
    return reduce128(a * b, mulhi(a, b));
#endif
}

GL_HD uint64_t from_i64(int64_t v) { return v >= 0 ? (uint64_t)v : GL_Q - (uint64_t)(-v); }

// multiply by a small non-negative integer s < 2^31
GL_HD uint64_t mul_small(uint64_t a, uint32_t s) { return reduce128(a * (uint64_t)s, mulhi(a, (uint64_t)s)); }

GL_HD uint64_t pow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mul(r, a);
        a = mul(a, a);
        e >>= 1;
    }
    return r;
}
GL_HD uint64_t inv(uint64_t a) { return pow(a, GL_Q - 2); }

struct K {
    uint64_t re, im;
};

GL_HD K kmk(uint64_t re, uint64_t im) { K r; r.re = re; r.im = im; return r; }
GL_HD K kzero() { return kmk(0, 0); }
GL_HD K kone() { return kmk(1, 0); }
GL_HD K kfq(uint64_t a) { return kmk(a, 0); }
GL_HD K kadd(K a, K b) { return kmk(add(a.re, b.re), add(a.im, b.im)); }
GL_HD K ksub(K a, K b) { return kmk(sub(a.re, b.re), sub(a.im, b.im)); }
GL_HD K kneg(K a) { return kmk(neg(a.re), neg(a.im)); }
GL_HD K kdbl(K a) { return kadd(a, a); }
GL_HD bool kiszero(K a) { return (a.re | a.im) == 0; }

// 7x mod q for any x < 2^64, canonical: 7x = 8x - x as a 67-bit value
// (lo, hi) with hi < 7, then lo + hi (2^32 - 1)
GL_HD uint64_t mul7(uint64_t x) {
    const uint64_t lo8 = x << 3;
    const uint64_t lo = lo8 - x;
    const uint64_t hi = (x >> 61) - (uint64_t)(lo8 < x);
    const uint64_t t1 = (hi << 32) - hi;
    uint64_t s = lo + t1;
    s += (uint64_t)(s < t1) * GL_EPS;  // a carry leaves s < t1 < 2^35
    return canon(s);
}

GL_HD K kmul(K a, K b) {
    uint64_t rr = add(mul(a.re, b.re), mul7(mul(a.im, b.im)));
    uint64_t ii = add(mul(a.re, b.im), mul(a.im, b.re));
    return kmk(rr, ii);
}
GL_HD K ksqr(K a) {
    uint64_t x = mul(a.re, a.im);
    return kmk(add(mul(a.re, a.re), mul7(mul(a.im, a.im))), add(x, x));
}
GL_HD K kscale(K a, uint64_t s) { return kmk(mul(a.re, s), mul(a.im, s)); }
// multiply by a small signed integer |s| < 2^31
GL_HD K kscale_small(K a, int32_t s) {
    if (s >= 0) return kmk(mul_small(a.re, (uint32_t)s), mul_small(a.im, (uint32_t)s));
    return kneg(kmk(mul_small(a.re, (uint32_t)(-s)), mul_small(a.im, (uint32_t)(-s))));
}
GL_HD K kinv(K a) {
    uint64_t n = sub(mul(a.re, a.re), mul7(mul(a.im, a.im)));
    uint64_t ni = inv(n);
    return kmk(mul(a.re, ni), mul(neg(a.im), ni));
}
// a + (b - a) * r
GL_HD K klerp(K a, K b, K r) { return kadd(a, kmul(ksub(b, a), r)); }

#ifdef __CUDACC__
// Unreduced sums of 64 x 64-bit products.  A 160-bit accumulator (five
// 32-bit words, little-endian) adds each 128-bit product with three carry
// chains and holds at least 2^32 products exactly; the sum is reduced mod q
// once, when it is read.
struct Acc160 {
    uint32_t w0, w1, w2, w3, w4;
};
__device__ __forceinline__ void acc_zero(Acc160& a) { a.w0 = a.w1 = a.w2 = a.w3 = a.w4 = 0; }
__device__ __forceinline__ void acc_mad(Acc160& a, uint64_t x, uint64_t y) {
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32), y0 = (uint32_t)y, y1 = (uint32_t)(y >> 32);
    // x y = x0 y0 + (x0 y1 + x1 y0) 2^32 + x1 y1 2^64
    asm("{\n\t"
        "mad.lo.cc.u32 %0, %5, %7, %0;\n\t"
        "madc.hi.cc.u32 %1, %5, %7, %1;\n\t"
        "madc.lo.cc.u32 %2, %6, %8, %2;\n\t"
        "madc.hi.cc.u32 %3, %6, %8, %3;\n\t"
        "addc.u32 %4, %4, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %8, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %8, %2;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.u32 %4, %4, 0;\n\t"
        "mad.lo.cc.u32 %1, %6, %7, %1;\n\t"
        "madc.hi.cc.u32 %2, %6, %7, %2;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.u32 %4, %4, 0;\n\t"
        "}"
        : "+r"(a.w0), "+r"(a.w1), "+r"(a.w2), "+r"(a.w3), "+r"(a.w4)
        : "r"(x0), "r"(x1), "r"(y0), "r"(y1));
}
// value mod q: 2^64 = 2^32 - 1, 2^96 = -1, 2^128 = -2^32 (mod q)
__device__ __forceinline__ uint64_t acc_reduce(const Acc160& a) {
    const uint64_t L = ((uint64_t)a.w1 << 32) | a.w0;
    const uint64_t B = ((uint64_t)a.w2 << 32) - a.w2;
    const uint64_t C = ((uint64_t)a.w4 << 32) | a.w3;
    return sub(add(canon(L), canon(B)), canon(C));
}
// Unreduced sum of K products x y: re = sum (x.re y.re + (7 x.im) y.im),
// im = sum (x.re y.im + x.im y.re), with 7 x.im (mod q) supplied by the
// caller (it is shared by every product with the same x); 2^31 products at
// most.
struct KAcc {
    Acc160 re, im;
};
__device__ __forceinline__ void kacc_zero(KAcc& a) { acc_zero(a.re); acc_zero(a.im); }
__device__ __forceinline__ void kacc_mad(KAcc& a, K x, uint64_t x7im, K y) {
    acc_mad(a.re, x.re, y.re);
    acc_mad(a.re, x7im, y.im);
    acc_mad(a.im, x.re, y.im);
    acc_mad(a.im, x.im, y.re);
}
__device__ __forceinline__ K kacc_reduce(const KAcc& a) { return kmk(acc_reduce(a.re), acc_reduce(a.im)); }
#endif

}  // namespace gl
