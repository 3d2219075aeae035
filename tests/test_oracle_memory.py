"""Pin the Twist / Shout oracle restatement (sparse, as the reference computes
it) against an independent dense restatement, round by round, and check the
sum-check relations the reference's own tests rely on (p(0)+p(1) equals the
running claim; the last round's constant equals the folded product)."""
import numpy as np
import pytest

import oracle
from memcase import kind_cols, rand_k, shout, trace
from pyref import K0, DenseMemSum, kadd, kmul

KINDS = {0: "shout_value", 1: "shout_adapter", 2: "bitness", 3: "twist_read", 4: "twist_write",
         5: "val_eval", 6: "total_inc", 7: "product"}


def tk(a):
    return (int(a[0]), int(a[1]))


def tcol(col):
    return [tk(v) for v in col]


def build(kind, ell, A, seed, general=False):
    c, rng = trace(ell, A, active=(3 << ell) // 4, seed=seed, general=general)
    s, _ = shout(ell, A, active=(3 << ell) // 4, seed=seed + 1)
    r_point = rand_k(rng, ell)
    r_addr = rand_k(rng, A)
    init = rand_k(rng, 1)[0]
    weights = None
    if kind == 2:
        cols = np.concatenate([c["ra_bits"], c["wa_bits"], c["has_read"][None]])
        weights = rand_k(rng, cols.shape[0])
    elif kind == 7:
        cols = rand_k(rng, 3 * (1 << ell)).reshape(3, 1 << ell, 2)
        cols[1, ::3] = 0
    else:
        cols = kind_cols(kind, c, s)
    if kind in (6, 7):
        r_point = None
    if kind not in (1, 3, 4, 5, 6):
        r_addr = None
    return cols, r_point, r_addr, (init if kind in (3, 4) else None), weights


def dense_of(kind, cols, r_point, r_addr, init, weights):
    return DenseMemSum(kind, [tcol(col) for col in cols],
                       None if r_point is None else tcol(r_point),
                       None if r_addr is None else tcol(r_addr),
                       K0 if init is None else tk(init),
                       None if weights is None else tcol(weights))


@pytest.mark.parametrize("general", [False, True])
@pytest.mark.parametrize("kind", sorted(KINDS))
def test_mem_oracle_matches_dense(kind, general):
    ell, A = 5, 3
    cols, r_point, r_addr, init, weights = build(kind, ell, A, seed=100 + kind, general=general)
    o = oracle.MemOracle(kind, cols, r_point, r_addr, init, weights)
    d = dense_of(kind, cols, r_point, r_addr, init, weights)
    assert tk(o.claim) == d.total()
    assert o.num_rounds() == ell
    deg = o.degree_bound()
    xs = np.array([[x, 0] for x in range(deg + 1)], np.uint64)
    rng = np.random.default_rng(7 + kind)
    claim = tk(o.claim)
    for rnd in range(ell):
        ys = o.evals_at(xs)
        assert [tk(y) for y in ys] == d.evals([(x, 0) for x in range(deg + 1)]), f"round {rnd}"
        assert kadd(tk(ys[0]), tk(ys[1])) == claim, f"p(0)+p(1) != claim at round {rnd}"
        r = rand_k(rng, 1)[0]
        # next claim = p(r), by Lagrange interpolation through the deg+1 points
        claim = tk(oracle.poly_eval_k(oracle.interpolate(xs, ys), r))
        o.fold(r)
        d.fold(tk(r))
    assert o.num_rounds() == 0
    fin = o.evals_at(xs[:2])
    assert tk(fin[0]) == claim
    assert [tk(v) for v in fin] == d.evals([(0, 0), (1, 0)])


def test_addr_lookup_claim():
    ell, A = 6, 4
    s, rng = shout(ell, A, active=50, seed=3)
    r_cycle = rand_k(rng, ell)
    w, claim = oracle.addr_lookup_weights(r_cycle, s["has_lookup"], s["addr_bits"], s["table"])
    chi = oracle.chi_table(r_cycle)
    want = K0
    bits = s["addr_bits"][:, :, 0].astype(np.int64)
    for t in range(1 << ell):
        if s["has_lookup"][t, 0]:
            a = sum(int(bits[b, t]) << b for b in range(A))
            want = kadd(want, kmul(tk(chi[t]), tk(s["table"][a])))
    assert tk(claim) == want
    # the same sum as the Shout value time-lane claim for an honest val column
    sv = oracle.MemOracle(0, kind_cols(0, None, s), r_cycle)
    assert tk(sv.claim) == want
    # the product oracle over [table, weights] starts from that claim
    prod = oracle.MemOracle(7, np.stack([s["table"], w]))
    assert tk(prod.claim) == want


def test_mem_oracle_empty_and_single():
    # ell = 0: no rounds, evals are the constant product
    cols = rand_k(np.random.default_rng(1), 2).reshape(2, 1, 2)
    o = oracle.MemOracle(7, cols)
    assert o.num_rounds() == 0
    v = o.evals_at(np.array([[0, 0], [5, 0]], np.uint64))
    assert tk(v[0]) == tk(v[1]) == kmul(tk(cols[0, 0]), tk(cols[1, 0]))
    # all-zero gate column: claim and every round are zero
    ell, A = 4, 2
    c, rng = trace(ell, A, active=0, seed=5)
    o = oracle.MemOracle(3, kind_cols(3, c), rand_k(rng, ell), rand_k(rng, A), rand_k(rng, 1)[0])
    assert tk(o.claim) == K0
    assert all(tk(y) == K0 for y in o.evals_at(np.array([[x, 0] for x in range(6)], np.uint64)))


def _init_at(init, r_addr):
    """eval_init_at_r_addr (neo-memory/src/mem_init.rs:133-163)."""
    acc = K0
    for a, v in init:
        chi = (1, 0)
        for b, rb in enumerate(r_addr):
            rb = tk(rb)
            chi = kmul(chi, rb if (a >> b) & 1 else ((1 - rb[0]) % Q, (-rb[1]) % Q))
        acc = kadd(acc, kmul((v % Q, 0), chi))
    return acc


Q = (1 << 64) - (1 << 32) + 1


@pytest.mark.parametrize("kind", [0, 1])
def test_twist_addr_lane_hands_over_to_time_lane(kind):
    """An honest trace: the address-lane sum is zero, and after ell_addr rounds
    its running claim equals the time-lane check's hypercube sum at r_addr."""
    ell, A = 6, 3
    c, rng = trace(ell, A, active=48, seed=21 + kind)
    r_cycle = rand_k(rng, ell)
    cols = kind_cols(3 if kind == 0 else 4, c)
    o = oracle.TwistAddrOracle(kind, cols, r_cycle, A, [(a, (v, 0)) for a, v in c["init"]])
    xs = np.array([[0, 0], [1, 0], [2, 0]], np.uint64)
    claim = K0
    chals = []
    for rnd in range(A):
        ys = o.evals_at(xs)
        assert kadd(tk(ys[0]), tk(ys[1])) == claim, f"round {rnd}"
        r = rand_k(rng, 1)[0]
        claim = tk(oracle.poly_eval_k(oracle.interpolate(xs, ys), r))
        o.fold(r)
        chals.append(r)
    assert o.num_rounds() == 0
    assert tk(o.evals_at(xs[:1])[0]) == claim
    init_r = _init_at(c["init"], chals)
    t = oracle.MemOracle(3 if kind == 0 else 4, cols, r_cycle, np.array(chals), np.array(init_r, np.uint64))
    assert tk(t.claim) == claim


def test_bus_openings_match_definition():
    rng = np.random.default_rng(4)
    m, chunk, ncols, m_in, ell = 256, 8, 5, 2, 8
    Z = rng.integers(-1, 2, size=(54, m)).astype(np.int8)
    r = rand_k(rng, ell)
    base = m - ncols * chunk
    y, ysc = oracle.bus_openings(Z, base, chunk, ncols, m_in, r)
    chi = oracle.chi_table(r)
    for cidx in range(ncols):
        sc = K0
        for rho in range(54):
            acc = K0
            for j in range(chunk):
                z = int(Z[rho, base + cidx * chunk + j]) % Q
                acc = kadd(acc, kmul(tk(chi[m_in + j]), (z, 0)))
            assert tk(y[cidx, rho]) == acc
            sc = kadd(sc, kmul(acc, (pow(2, rho, Q), 0)))
        assert tk(ysc[cidx]) == sc
