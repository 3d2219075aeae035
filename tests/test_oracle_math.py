"""Pins the C oracle's arithmetic, commitment, decomposition and RLC/DEC
against independent Python-integer restatements and the reference's
relational tests (crates/neo-math/tests, crates/neo-ajtai/tests)."""
import numpy as np
import pytest

import oracle as O
from tests import pyref

Q = pyref.Q


def test_fq_mul_matches_bigint():
    rng = np.random.default_rng(1)
    a = rng.integers(0, Q, size=4000, dtype=np.uint64)
    b = rng.integers(0, Q, size=4000, dtype=np.uint64)
    edge = np.array([0, 1, Q - 1, Q - 2, 2**32, 2**32 - 1, 2**63, 2**64 - 2**32], dtype=np.uint64)
    a = np.concatenate([a, edge, edge[::-1]])
    b = np.concatenate([b, edge[::-1], edge])
    r = O.fq_mul(a, b)
    assert all(int(r[i]) == int(a[i]) * int(b[i]) % Q for i in range(a.size))


def test_k_mul_and_inverse():
    rng = np.random.default_rng(2)
    a = rng.integers(0, Q, size=(500, 2), dtype=np.uint64)
    b = rng.integers(0, Q, size=(500, 2), dtype=np.uint64)
    r = O.k_mul(a, b)
    for i in range(500):
        assert tuple(int(x) for x in r[i]) == pyref.kmul((int(a[i, 0]), int(a[i, 1])), (int(b[i, 0]), int(b[i, 1])))
    inv = np.empty_like(a)
    O.lib().or_k_inv_batch(O.ptr(a), 500, O.ptr(inv))
    one = O.k_mul(a, inv)
    assert np.all(one[:, 0] == 1) and np.all(one[:, 1] == 0)


def test_rq_mul_matches_polynomial_division():
    rng = np.random.default_rng(3)
    for _ in range(20):
        a = rng.integers(0, Q, size=54, dtype=np.uint64)
        b = rng.integers(0, Q, size=54, dtype=np.uint64)
        assert [int(x) for x in O.rq_mul(a, b)] == pyref.rq_mul([int(x) for x in a], [int(x) for x in b])


def test_rot_matrix_columns_are_monomial_products():
    # rot(a) column j = cf(a * X^j mod Phi_81) (crates/neo-math/src/s_action.rs:27-41)
    rng = np.random.default_rng(4)
    a = rng.integers(-2, 3, size=54).astype(np.int8)
    R = O.rot_matrix(a)
    for j in range(54):
        mono = [0] * 54
        mono[j] = 1
        assert [int(x) for x in R[:, j]] == pyref.rq_mul([int(x) % Q for x in a], mono)


def test_commit_matches_ring_definition():
    rng = np.random.default_rng(5)
    kappa, m = 3, 5
    pp = rng.integers(0, Q, size=(kappa, m, 54), dtype=np.uint64)
    Z = rng.integers(-1, 2, size=(54, m)).astype(np.int8)
    c = O.commit_digits(pp, Z, threads=1)
    ref = pyref.commit(pp.tolist(), [[int(x) % Q for x in row] for row in Z.tolist()])
    assert [[int(x) for x in row] for row in c] == ref


def test_commit_digit_path_equals_general_path():
    rng = np.random.default_rng(6)
    kappa, m = 4, 300
    pp = rng.integers(0, Q, size=(kappa, m, 54), dtype=np.uint64)
    Z = rng.integers(-1, 2, size=(54, m)).astype(np.int8)
    Zf = np.where(Z < 0, np.uint64(Q - 1), Z.astype(np.uint64))
    assert np.array_equal(O.commit_digits(pp, Z), O.commit_fq(pp, Zf))


def test_commit_s_homomorphism():
    # rho * L(Z) = L(rho Z) (crates/neo-ajtai/tests/s_homomorphism.rs)
    rng = np.random.default_rng(7)
    kappa, m = 2, 8
    pp = rng.integers(0, Q, size=(kappa, m, 54), dtype=np.uint64)
    Z = rng.integers(-1, 2, size=(54, m)).astype(np.int8)
    rho = rng.integers(-2, 3, size=54).astype(np.int8)
    Zf = np.where(Z < 0, np.uint64(Q - 1), Z.astype(np.uint64))
    R = O.rot_matrix(rho)
    RZ = np.array([[sum(int(R[r, k]) * int(Zf[k, c]) for k in range(54)) % Q for c in range(m)] for r in range(54)],
                  dtype=np.uint64)
    lhs = O.commit_fq(pp, RZ)
    c = O.commit_fq(pp, Zf)
    rhs = np.array([O.rq_mul(np.array([int(x) % Q for x in rho], np.uint64), c[i]) for i in range(kappa)])
    assert np.array_equal(lhs, rhs)


def test_decomp_roundtrip_and_range():
    rng = np.random.default_rng(8)
    z = rng.integers(0, 1 << 32, size=1000, dtype=np.uint64)
    neg = (Q - rng.integers(1, 1 << 40, size=1000, dtype=np.uint64)).astype(np.uint64)
    z = np.concatenate([z, neg, np.array([0, 1, Q - 1, (1 << 53) - 1], np.uint64)])
    Z = O.decomp_b2(z)
    assert Z.shape == (54, z.size)
    assert set(np.unique(Z)).issubset({-1, 0, 1})
    assert np.array_equal(O.recompose_b2(Z), z)


def test_decomp_representability_limit():
    # values with balanced magnitude >= 2^54 do not recompose
    # (crates/neo-ajtai/tests/decomp_representability_limit.rs)
    z = np.array([1 << 54, (1 << 60) + 5], np.uint64)
    assert not np.array_equal(O.recompose_b2(O.decomp_b2(z)), z)


def test_split_b_roundtrip_and_error():
    rng = np.random.default_rng(9)
    Zmix = rng.integers(-4095, 4096, size=(54, 64)).astype(np.int32)
    planes, nz = O.split_b(Zmix, 12, 2)
    rec = sum((2 ** i) * planes[i].astype(np.int64) for i in range(12))
    assert np.array_equal(rec, Zmix)
    assert set(np.unique(planes)).issubset({-1, 0, 1})
    assert nz.all()
    with pytest.raises(ValueError):
        O.split_b(np.array([[4096]], np.int32), 12, 2)


def test_rlc_mix_matches_rot_products():
    rng = np.random.default_rng(10)
    count, m = 3, 16
    rho = rng.integers(-2, 3, size=(count, 54)).astype(np.int8)
    Zs = rng.integers(-1, 2, size=(count, 54, m)).astype(np.int8)
    mix = O.rlc_mix(rho, Zs)
    ref = np.zeros((54, m), dtype=object)
    for i in range(count):
        R = O.rot_matrix(rho[i]).astype(object)
        Rs = np.where(R > Q // 2, R - Q, R)
        ref = ref + Rs.dot(Zs[i].astype(object))
    assert np.array_equal(mix.astype(object), ref)
    # count == 1 is the identity
    assert np.array_equal(O.rlc_mix(rho[:1], Zs[:1]), Zs[0].astype(np.int32))


def test_interpolate_roundtrip():
    rng = np.random.default_rng(11)
    xs = np.array([[i, 0] for i in range(7)], np.uint64)
    ys = rng.integers(0, Q, size=(7, 2), dtype=np.uint64)
    co = O.interpolate(xs, ys)
    for i in range(7):
        assert np.array_equal(O.poly_eval_k(co, xs[i]), ys[i])
