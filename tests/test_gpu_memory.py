"""Twist / Shout time-lane oracles on the GPU against the oracle restatement,
bit for bit, every round; and at the single-shard-with-memory sizes (time
domain 2^16, 2^14 active steps, Twist 2^12 cells, Shout 2^16 table) through
size-independent properties: every round's p(0)+p(1) equals the running claim
and the last round's constant equals the product of the columns' multilinear
extensions at the challenge point."""
import numpy as np
import pytest

import oracle
from memcase import (eq_bit_np, excl_prefix_np, kadd_np, kind_cols, ksub_np, mle_eval, rand_k, shout, trace)
from nightstream_b200 import gpu

pytestmark = pytest.mark.gpu


def case(kind, ell, A, seed, general=False, active=None):
    active = (3 << ell) // 4 if active is None else active
    c, rng = trace(ell, A, active=active, seed=seed, general=general)
    s, _ = shout(ell, A, active=active, seed=seed + 1)
    r_point, r_addr, init = rand_k(rng, ell), rand_k(rng, A), rand_k(rng, 1)[0]
    weights = None
    if kind == 2:
        cols = np.concatenate([c["ra_bits"], c["wa_bits"], c["has_read"][None]])
        weights = rand_k(rng, cols.shape[0])
    elif kind == 7:
        cols = rand_k(rng, 3 << ell).reshape(3, 1 << ell, 2)
    else:
        cols = kind_cols(kind, c, s)
    if kind in (6, 7):
        r_point = None
    if kind not in (1, 3, 4, 5, 6):
        r_addr = None
    return cols, r_point, r_addr, (init if kind in (3, 4) else None), weights, c, s, rng


@pytest.mark.parametrize("general", [False, True])
@pytest.mark.parametrize("kind", range(8))
def test_mem_oracle_gpu_matches_oracle(ctx, kind, general):
    ell, A = 10, 4
    cols, r_point, r_addr, init, weights, _, _, rng = case(kind, ell, A, 300 + kind, general)
    ref = oracle.MemOracle(kind, cols, r_point, r_addr, init, weights)
    g = gpu.GpuMemOracle(ctx, kind, cols, r_point, r_addr, init, weights)
    assert np.array_equal(g.claim, ref.claim)
    assert g.num_rounds() == ref.num_rounds() == ell
    assert g.degree_bound() == ref.degree_bound()
    xs = np.array([[x, 0] for x in range(g.degree_bound() + 1)] + [[123456789, 987654321]], np.uint64)
    for rnd in range(ell + 1):
        assert np.array_equal(g.evals_at(xs), ref.evals_at(xs)), f"round {rnd}"
        if rnd < ell:
            r = rand_k(rng, 1)[0]
            g.fold(r)
            ref.fold(r)
    assert g.num_rounds() == 0
    g.close()


@pytest.mark.parametrize("kind", [0, 1, 3, 4, 5, 6])
def test_mem_oracle_gpu_full_size(ctx, kind):
    """Time domain 2^16 with 2^14 active steps; Twist 2^12 cells (ell_addr 12),
    Shout 2^16-entry table (ell_addr 16)."""
    ell = 16
    A = 16 if kind in (0, 1) else 12
    cols, r_point, r_addr, init, weights, c, s, rng = case(kind, ell, A, 900 + kind, active=1 << 14)
    g = gpu.GpuMemOracle(ctx, kind, cols, r_point, r_addr, init, weights)
    deg = g.degree_bound()
    xs = np.array([[x, 0] for x in range(deg + 1)], np.uint64)
    claim = g.claim.copy()
    chals = []
    for rnd in range(ell):
        ys = g.evals_at(xs)
        assert np.array_equal(kadd_np(ys[0], ys[1]), claim), f"round {rnd}"
        r = rand_k(rng, 1)[0]
        claim = oracle.poly_eval_k(oracle.interpolate(xs, ys), r)
        g.fold(r)
        chals.append(r)
    fin = g.evals_at(xs[:1])[0]
    assert np.array_equal(fin, claim)
    pt = np.array(chals)
    one = np.array([1, 0], np.uint64)
    k = lambda a, b: oracle.k_mul(np.asarray(a, np.uint64).reshape(-1, 2), np.asarray(b, np.uint64).reshape(-1, 2))[0]

    def eqpt(a, b):  # Π_i eq(a_i, b_i)
        acc = one
        for ai, bi in zip(a, b):
            acc = k(acc, kadd_np(k(ai, bi), k(ksub_np(one, ai), ksub_np(one, bi))))
        return acc

    def eqbits(bitcols):
        acc = one
        for b in range(A):
            acc = k(acc, eq_bit_np(oracle, mle_eval(oracle, bitcols[b], pt)[None], r_addr[b])[0])
        return acc

    if kind == 0:
        want = k(k(eqpt(r_point, pt), mle_eval(oracle, cols[0], pt)), mle_eval(oracle, cols[1], pt))
    elif kind == 1:
        want = k(k(eqpt(r_point, pt), mle_eval(oracle, cols[0], pt)), eqbits(cols[1:]))
    elif kind in (3, 4):
        terms = oracle.k_mul(c["has_write"], c["inc"])
        for b in range(A):
            terms = oracle.k_mul(terms, eq_bit_np(oracle, c["wa_bits"][b], r_addr[b]))
        vp = mle_eval(oracle, excl_prefix_np(init, terms), pt)
        if kind == 3:
            diff = ksub_np(vp, mle_eval(oracle, c["rv"], pt))
            want = k(k(k(eqpt(r_point, pt), mle_eval(oracle, c["has_read"], pt)), diff), eqbits(c["ra_bits"]))
        else:
            delta = ksub_np(ksub_np(mle_eval(oracle, c["wv"], pt), vp), mle_eval(oracle, c["inc"], pt))
            want = k(k(k(eqpt(r_point, pt), mle_eval(oracle, c["has_write"], pt)), delta), eqbits(c["wa_bits"]))
    else:
        want = k(k(mle_eval(oracle, c["has_write"], pt), mle_eval(oracle, c["inc"], pt)), eqbits(c["wa_bits"]))
        if kind == 5:
            # LT(pt, r_time) (neo-memory/src/mle.rs:7-24)
            lt = np.zeros(2, np.uint64)
            for i in range(ell):
                tail = one
                for j in range(i + 1, ell):
                    tail = k(tail, kadd_np(k(pt[j], r_point[j]), k(ksub_np(one, pt[j]), ksub_np(one, r_point[j]))))
                lt = kadd_np(lt, k(k(ksub_np(one, pt[i]), r_point[i]), tail))
            want = k(want, lt)
    assert np.array_equal(fin, want)
    g.close()


def test_addr_lookup_weights_gpu(ctx):
    for ell, A, active in ((10, 6, 700), (16, 16, 1 << 14)):
        s, rng = shout(ell, A, active=active, seed=ell)
        r_cycle = rand_k(rng, ell)
        w_ref, c_ref = oracle.addr_lookup_weights(r_cycle, s["has_lookup"], s["addr_bits"], s["table"])
        w, c = gpu.addr_lookup_weights(ctx, r_cycle, s["has_lookup"], s["addr_bits"], s["table"])
        assert np.array_equal(w, w_ref) and np.array_equal(c, c_ref)
        if ell == 16:
            # the address rounds: PRODUCT over [table, weights] starts from the same claim
            p = gpu.GpuMemOracle(ctx, gpu.MEM_PRODUCT, np.stack([s["table"], w]))
            assert np.array_equal(p.claim, c)
            p.close()


def test_mem_oracle_gpu_errors(ctx):
    cols = np.zeros((3, 16, 2), np.uint64)
    with pytest.raises(gpu.NeoGpuError) as e:
        gpu.GpuMemOracle(ctx, gpu.MEM_SHOUT_VALUE, cols, rand_k(np.random.default_rng(0), 4))
    assert e.value.code == 1
    # ell = 0: no rounds, the constant product
    one = np.array([[[5, 1]], [[7, 0]]], np.uint64)
    p = gpu.GpuMemOracle(ctx, gpu.MEM_PRODUCT, one)
    assert p.num_rounds() == 0
    assert np.array_equal(p.evals_at(np.array([[0, 0], [9, 9]], np.uint64)),
                          np.array([[35, 7], [35, 7]], np.uint64))
    p.close()


def test_bitness_without_columns(ctx):
    """LazyWeightedBitnessOracleSparseTime with no columns sums to zero (twist_oracle.rs:545-548)."""
    r = rand_k(np.random.default_rng(2), 5)
    g = gpu.GpuMemOracle(ctx, gpu.MEM_BITNESS, np.zeros((0, 32, 2), np.uint64), r, weights=np.zeros((0, 2), np.uint64))
    assert np.array_equal(g.claim, np.zeros(2, np.uint64))
    assert not g.evals_at(np.array([[0, 0], [3, 0]], np.uint64)).any()
    g.close()


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("general", [False, True])
def test_twist_addr_gpu_matches_oracle(ctx, kind, general):
    ell, A = 10, 6
    c, rng = trace(ell, A, active=700, seed=50 + kind, general=general)
    r_cycle = rand_k(rng, ell)
    cols = kind_cols(3 if kind == 0 else 4, c)
    init = [(a, (v, 0)) for a, v in c["init"][:40]]
    ref = oracle.TwistAddrOracle(kind, cols, r_cycle, A, init)
    g = gpu.GpuTwistAddrOracle(ctx, kind, cols, r_cycle, A, init)
    xs = np.array([[0, 0], [1, 0], [2, 0], [77, 5]], np.uint64)
    for rnd in range(A + 1):
        assert np.array_equal(g.evals_at(xs), ref.evals_at(xs)), f"round {rnd}"
        if rnd < A:
            r = rand_k(rng, 1)[0]
            g.fold(r)
            ref.fold(r)
    assert g.num_rounds() == 0
    g.close()


def test_twist_addr_gpu_full_size(ctx):
    """Twist 2^12 cells, 2^14 events in a 2^16 time domain: the address lane
    sums to zero for an honest trace and hands over to the time-lane claim."""
    ell, A = 16, 12
    c, rng = trace(ell, A, active=1 << 14, seed=77)
    r_cycle = rand_k(rng, ell)
    init = [(a, (v, 0)) for a, v in c["init"]]
    for kind in (0, 1):
        cols = kind_cols(3 if kind == 0 else 4, c)
        g = gpu.GpuTwistAddrOracle(ctx, kind, cols, r_cycle, A, init)
        xs = np.array([[0, 0], [1, 0], [2, 0]], np.uint64)
        claim = np.zeros(2, np.uint64)
        chals = []
        for rnd in range(A):
            ys = g.evals_at(xs)
            assert np.array_equal(kadd_np(ys[0], ys[1]), claim), f"kind {kind} round {rnd}"
            r = rand_k(rng, 1)[0]
            claim = oracle.poly_eval_k(oracle.interpolate(xs, ys), r)
            g.fold(r)
            chals.append(r)
        assert np.array_equal(g.evals_at(xs[:1])[0], claim)
        # time-lane check at r_addr starts from the address lane's final value
        init_r = np.zeros(2, np.uint64)
        chi_addr = oracle.chi_table(np.array(chals))
        for a, (v, _) in init:
            init_r = kadd_np(init_r, oracle.k_mul(np.array([[v, 0]], np.uint64), chi_addr[a:a + 1])[0])
        t = gpu.GpuMemOracle(ctx, 3 if kind == 0 else 4, cols, r_cycle, np.array(chals), init_r)
        assert np.array_equal(t.claim, claim)
        t.close()
        g.close()
