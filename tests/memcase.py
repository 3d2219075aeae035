"""Seeded Twist / Shout time-lane instances shared by the CPU and GPU tests.

A RISC-V-style memory trace: per step one read and one write of a 2^ell_addr
cell memory (addresses 70% stride-4 sequential, 30% uniform), read values from
the current memory, write increments inc = wv - mem[wa]; a Shout lookup per
step into a uniform table. Columns are K elements stored as uint64 (re, im).
"""
import numpy as np

Q = (1 << 64) - (1 << 32) + 1


def rand_k(rng, n, base_only=False):
    re = rng.integers(0, Q, size=n, dtype=np.uint64)
    im = np.zeros(n, np.uint64) if base_only else rng.integers(0, Q, size=n, dtype=np.uint64)
    return np.stack([re, im], axis=-1)


def to_k(vals):
    v = np.asarray(vals, dtype=np.uint64)
    return np.stack([v, np.zeros_like(v)], axis=-1)


def bit_cols(addrs, ell_addr):
    a = np.asarray(addrs, dtype=np.uint64)
    return np.stack([to_k((a >> np.uint64(b)) & np.uint64(1)) for b in range(ell_addr)])


def trace(ell, ell_addr, active, seed, general=False):
    """Dense columns of one memory trace over a 2^ell time domain with
    `active` real steps. general=True replaces gates / bits by arbitrary K
    values at the active rows (the oracles are defined for any K column)."""
    rng = np.random.default_rng(seed)
    L, P = 1 << ell, 1 << ell_addr
    mem = [int(x) for x in rng.integers(0, 1 << 32, size=P)]
    init = [(a, mem[a]) for a in range(P) if mem[a]]
    has_r, has_w, ra, wa, rv, wv, inc = (np.zeros(L, np.uint64) for _ in range(7))
    pos = 0
    for t in range(active):
        if rng.random() < 0.7:
            pos = (pos + 4) % P
            a_r = pos
        else:
            a_r = int(rng.integers(0, P))
        a_w = (a_r + int(rng.integers(0, 2))) % P
        has_r[t] = 1 if rng.random() < 0.9 else 0
        has_w[t] = 1 if rng.random() < 0.8 else 0
        ra[t], wa[t] = a_r, a_w
        if has_r[t]:
            rv[t] = mem[a_r]
        if has_w[t]:
            v = int(rng.integers(0, 1 << 32))
            wv[t] = v
            inc[t] = (v - mem[a_w]) % Q
            mem[a_w] = v
        else:
            wa[t] = 0
    c = dict(has_read=to_k(has_r), has_write=to_k(has_w), rv=to_k(rv), wv=to_k(wv), inc=to_k(inc),
             ra_bits=bit_cols(ra * has_r, ell_addr), wa_bits=bit_cols(wa, ell_addr), init=init)
    if general:
        for key in ("has_read", "has_write"):
            g = c[key]
            nz = np.nonzero(g[:, 0])[0]
            g[nz] = rand_k(rng, len(nz))
        for key in ("ra_bits", "wa_bits"):
            for b in range(ell_addr):
                col = c[key][b]
                nz = np.nonzero(col[:, 0])[0]
                col[nz] = rand_k(rng, len(nz))
    return c, rng


def shout(ell, ell_addr, active, seed, table_len=None):
    rng = np.random.default_rng(seed)
    L, P = 1 << ell, 1 << ell_addr
    table = rand_k(rng, table_len or P, base_only=True)
    has = np.zeros(L, np.uint64)
    idx = np.zeros(L, np.uint64)
    for t in range(active):
        has[t] = 1 if rng.random() < 0.85 else 0
        idx[t] = int(rng.integers(0, P)) if has[t] else 0
    val = np.zeros((L, 2), np.uint64)
    val[:active] = table[idx[:active].astype(np.int64) % table.shape[0]]
    val[has == 0] = 0
    return dict(has_lookup=to_k(has), val=val, addr_bits=bit_cols(idx, ell_addr), table=table), rng


def kind_cols(kind, c, s=None):
    """Column stacks in the C ABI's order for each oracle kind."""
    if kind == 0:
        return np.stack([s["has_lookup"], s["val"]])
    if kind == 1:
        return np.concatenate([s["has_lookup"][None], s["addr_bits"]])
    if kind == 3:
        return np.concatenate([c["has_read"][None], c["rv"][None], c["ra_bits"], c["has_write"][None],
                               c["inc"][None], c["wa_bits"]])
    if kind == 4:
        return np.concatenate([c["has_write"][None], c["wv"][None], c["inc"][None], c["wa_bits"]])
    if kind in (5, 6):
        return np.concatenate([c["has_write"][None], c["inc"][None], c["wa_bits"]])
    raise ValueError(kind)


# --- vectorised K helpers for size-independent checks --------------------------
def _canon(x):
    q = np.uint64(Q)
    return np.where(x >= q, x - q, x)


def kadd_np(a, b):
    a, b = np.asarray(a, np.uint64), np.asarray(b, np.uint64)
    s = a + b
    s = s + (s < a).astype(np.uint64) * np.uint64(0xFFFFFFFF)
    return _canon(s)


def ksub_np(a, b):
    a, b = np.asarray(a, np.uint64), np.asarray(b, np.uint64)
    d = a - b
    return d + (a < b).astype(np.uint64) * np.uint64(Q)


def ksum_np(a):
    """Σ over axis 0 of a (n, 2) K array, exactly (32-bit halves)."""
    a = np.asarray(a, np.uint64)
    lo = (a & np.uint64(0xFFFFFFFF)).sum(axis=0, dtype=np.uint64)
    hi = (a >> np.uint64(32)).sum(axis=0, dtype=np.uint64)
    return np.array([(int(lo[i]) + (int(hi[i]) << 32)) % Q for i in range(2)], np.uint64)


def mle_eval(oracle_mod, col, point):
    """Multilinear extension of a K column at a K point (little-endian variables)."""
    chi = oracle_mod.chi_table(point)
    return ksum_np(oracle_mod.k_mul(chi, col).reshape(-1, 2))


def eq_bit_np(oracle_mod, col, u):
    """eq_bit_affine(col, u) = col·(2u−1) + (1−u), elementwise."""
    u = np.asarray(u, np.uint64)
    two_u_m1 = ksub_np(kadd_np(u, u), np.array([1, 0], np.uint64))
    one_m_u = ksub_np(np.array([1, 0], np.uint64), u)
    prod = oracle_mod.k_mul(np.asarray(col, np.uint64).reshape(-1, 2),
                            np.broadcast_to(two_u_m1, (col.shape[0], 2)).copy())
    return kadd_np(prod, one_m_u)


def excl_prefix_np(init, terms):
    re, im = int(init[0]), int(init[1])
    out = np.empty_like(terms)
    for t in range(terms.shape[0]):
        out[t, 0], out[t, 1] = re, im
        re = (re + int(terms[t, 0])) % Q
        im = (im + int(terms[t, 1])) % Q
    return out
