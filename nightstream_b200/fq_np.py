"""Vectorised Goldilocks (q = 2^64 - 2^32 + 1) arithmetic on numpy uint64.

Host-side helper for building seeded synthetic inputs (R1CS coefficients,
solved constraint rows).  The reduction uses 2^64 = 2^32 - 1 and
2^96 = -1 (mod q).
"""
import numpy as np

Q = np.uint64(0xFFFFFFFF00000001)
EPS = np.uint64(0xFFFFFFFF)
M32 = np.uint64(0xFFFFFFFF)
S32 = np.uint64(32)


def _u(x):
    return np.asarray(x, dtype=np.uint64)


def canon(a):
    a = _u(a)
    return np.where(a >= Q, a - Q, a)


def add(a, b):
    a, b = _u(a), _u(b)
    with np.errstate(over="ignore"):
        s = a + b
        carry = s < a
        s = s + np.where(carry, EPS, np.uint64(0))
    return canon(s)


def sub(a, b):
    a, b = _u(a), _u(b)
    with np.errstate(over="ignore"):
        return np.where(a >= b, a - b, a + (Q - b))


def neg(a):
    a = _u(a)
    return np.where(a == 0, np.uint64(0), Q - a)


def mul(a, b):
    a, b = np.broadcast_arrays(_u(a), _u(b))
    with np.errstate(over="ignore"):
        a0, a1 = a & M32, a >> S32
        b0, b1 = b & M32, b >> S32
        p00 = a0 * b0
        p01 = a0 * b1
        p10 = a1 * b0
        p11 = a1 * b1
        mid = p01 + p10
        mid_carry = (mid < p01).astype(np.uint64)
        lo = p00 + (mid << S32)
        lo_carry = (lo < p00).astype(np.uint64)
        hi = p11 + (mid >> S32) + (mid_carry << S32) + lo_carry
        hi_hi = hi >> S32
        hi_lo = hi & M32
        t0 = lo - hi_hi
        t0 = t0 - np.where(lo < hi_hi, EPS, np.uint64(0))
        t1 = hi_lo * EPS
        s = t0 + t1
        s = s + np.where(s < t0, EPS, np.uint64(0))
    return canon(s)


def pow_(a, e: int):
    a = _u(a).copy()
    r = np.ones_like(a)
    while e:
        if e & 1:
            r = mul(r, a)
        a = mul(a, a)
        e >>= 1
    return r


def inv(a):
    return pow_(a, (1 << 64) - (1 << 32) - 1)


def from_i64(v):
    v = np.asarray(v, dtype=np.int64)
    with np.errstate(over="ignore"):
        return np.where(v >= 0, v.astype(np.uint64), Q - (-v).astype(np.uint64))
