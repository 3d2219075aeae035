"""Seeded synthetic workloads with the shapes of the Neo hot-path benchmarks.

R1CS-shaped CCS over Goldilocks: n = m = 2^ell, 3 nonzeros per row of A and
B at seeded-uniform columns with uniform F_q coefficients; each row of C has
2 uniform entries plus one entry solved so that (Az)_r (Bz)_r = (Cz)_r.
The witness z is uniform in [0, 2^32) with z[0] = 1 (public constant one,
m_in = 1).  Values stay below 2^54 so that the b=2, d=54 decomposition
recomposes exactly (crates/neo-ajtai/src/decomp.rs:118-158).
"""
import numpy as np

from . import fq_np as F
from .ccs import CscMatrix, r1cs_to_ccs, CcsStructure
from .params import Q


def _distinct_cols(rng, n, m, k):
    cols = rng.integers(0, m, size=(n, k), dtype=np.int64)
    if m < 2 * k:
        return cols  # too few columns for distinct picks: duplicates add up
    while True:
        s = np.sort(cols, axis=1)
        dup = np.any(s[:, 1:] == s[:, :-1], axis=1)
        if not dup.any():
            return cols
        cols[dup] = rng.integers(0, m, size=(int(dup.sum()), k), dtype=np.int64)


def _uniform_fq(rng, shape):
    while True:
        v = rng.integers(0, 1 << 64, size=shape, dtype=np.uint64)
        bad = v >= np.uint64(Q)
        if not bad.any():
            return v
        v[bad] = rng.integers(0, 1 << 32, size=int(bad.sum()), dtype=np.uint64)
        return v


def make_r1cs(ell: int, seed: int, z_bits: int = 32, z: np.ndarray = None, max_col: int = None):
    """Return (ccs, z) for a satisfied random R1CS with n = m = 2^ell
    (z drawn here, or the given witness with z[0] = 1).  max_col: constraints
    only touch columns < max_col (any values beyond stay satisfying)."""
    n = m = 1 << ell
    rng = np.random.default_rng(seed)
    if z is None:
        z = rng.integers(0, 1 << z_bits, size=m, dtype=np.uint64)
        z[0] = 1
    else:
        z = np.asarray(z, dtype=np.uint64).copy()
        rng.integers(0, 1 << z_bits, size=m, dtype=np.uint64)  # keep the stream aligned
    mc = m if max_col is None else max_col
    a_cols = _distinct_cols(rng, n, mc, 3)
    b_cols = _distinct_cols(rng, n, mc, 3)
    c_cols = _distinct_cols(rng, n, mc, 3)
    # the solved column must hold a nonzero witness value
    zero = z[c_cols[:, 2]] == 0
    while zero.any():
        c_cols[zero, 2] = rng.integers(0, mc, size=int(zero.sum()))
        zero = z[c_cols[:, 2]] == 0
    a_vals = _uniform_fq(rng, (n, 3))
    b_vals = _uniform_fq(rng, (n, 3))
    c_vals = _uniform_fq(rng, (n, 3))

    def rowdot(cols, vals, k):
        acc = np.zeros(n, dtype=np.uint64)
        for q in range(k):
            acc = F.add(acc, F.mul(vals[:, q], z[cols[:, q]]))
        return acc

    az = rowdot(a_cols, a_vals, 3)
    bz = rowdot(b_cols, b_vals, 3)
    partial = rowdot(c_cols, c_vals, 2)
    target = F.sub(F.mul(az, bz), partial)
    c_vals[:, 2] = F.mul(target, F.inv(z[c_cols[:, 2]]))
    rows = np.repeat(np.arange(n, dtype=np.int64), 3)
    A = CscMatrix.from_coo(n, m, rows, a_cols.reshape(-1), a_vals.reshape(-1))
    B = CscMatrix.from_coo(n, m, rows, b_cols.reshape(-1), b_vals.reshape(-1))
    C = CscMatrix.from_coo(n, m, rows, c_cols.reshape(-1), c_vals.reshape(-1))
    return r1cs_to_ccs(n, m, A, B, C), z


def check_r1cs(ccs: CcsStructure, z: np.ndarray) -> bool:
    """(Az) o (Bz) == Cz over F_q."""
    outs = []
    for M in ccs.matrices[1:4]:
        row_ptr, cols, vals = M.to_csr()
        prod = F.mul(vals, z[cols])
        acc = np.zeros(ccs.n, dtype=np.uint64)
        rp = row_ptr.astype(np.int64)
        for q in range(3):
            acc = F.add(acc, prod[rp[:-1] + q])
        outs.append(acc)
    return bool(np.all(F.mul(outs[0], outs[1]) == outs[2]))


def uniform_k(rng, count: int) -> np.ndarray:
    """count uniform K = F_q[u]/(u^2-7) elements as [count, 2] uint64."""
    return _uniform_fq(rng, (count, 2))


def memory_trace(steps: int, shout_ell, twist_ell, seed: int, table_len: int = None, init_cells: int = 64,
                 lookup_rate: float = 1.0, rw_rate: float = 1.0):
    """One fold step's worth of a RISC-V-style trace: per step a Shout lookup
    (probability lookup_rate; uniform index into a table of uniform 32-bit
    entries) and a Twist read + write (probability rw_rate each; addresses 70 %
    stride-4 sequential / 30 % uniform over 2^twist_ell cells, 32-bit values;
    the first init_cells cells start nonzero, 0 = MemInit::Zero).  shout_ell /
    twist_ell: one int per instance (or a single int).  Returns the bus columns
    (values per step, Shout instances first then Twist, in the shared-bus
    column order) and the instance data."""
    buses, mem, _ = memory_trace_chunks(1, steps, shout_ell, twist_ell, seed, table_len, init_cells, lookup_rate,
                                        rw_rate)
    return buses[0], mem


def memory_trace_chunks(n_chunks: int, steps: int, shout_ell, twist_ell, seed: int, table_len: int = None,
                        init_cells: int = 64, lookup_rate: float = 1.0, rw_rate: float = 1.0):
    """A trace of n_chunks * steps steps (as memory_trace) split into fold
    steps of `steps` trace steps.  Returns the per-chunk bus columns, the
    instance data (with the initial state of chunk 0) and, per chunk, the
    MemInit of every Twist instance: the nonzero cells at the chunk's start in
    increasing address order (mem_init_from_state_map,
    crates/neo-memory/src/mem_init.rs:65-90)."""
    rng = np.random.default_rng(seed)
    shout_ells = [shout_ell] if isinstance(shout_ell, int) else list(shout_ell)
    twist_ells = [twist_ell] if isinstance(twist_ell, int) else list(twist_ell)
    S = n_chunks * steps
    cols, shout, twist = [], [], []
    inits = [[] for _ in range(n_chunks)]
    for se in shout_ells:
        tl = table_len or (1 << se)
        table = rng.integers(0, 1 << 32, size=tl, dtype=np.uint64)
        idx = rng.integers(0, tl, size=S)
        has = (rng.random(S) < lookup_rate).astype(np.int64)
        idx = idx * has
        for b in range(se):
            cols.append((idx >> b) & 1)
        cols.append(has)                               # has_lookup
        cols.append(table[idx] * has.astype(np.uint64))  # val
        shout.append(dict(ell_addr=se, k=1 << se, d=1, n_side=1 << se, ell=se, table=table))
    for te in twist_ells:
        P = 1 << te
        n0 = min(init_cells, P)
        init = [(int(a), int(v)) for a, v in zip(range(n0), rng.integers(1, 1 << 32, size=n0))]
        mem = np.zeros(P, dtype=object)
        for a, v in init:
            mem[a] = v
        ra = np.zeros(S, np.int64)
        wa = np.zeros(S, np.int64)
        hr = (rng.random(S) < rw_rate).astype(np.int64)
        hw = (rng.random(S) < rw_rate).astype(np.int64)
        rv = np.zeros(S, dtype=object)
        wv = rng.integers(0, 1 << 32, size=S) * hw
        inc = np.zeros(S, dtype=object)
        pos = 0
        for j in range(S):
            if j % steps == 0:
                inits[j // steps].append([(a, int(mem[a])) for a in range(P) if mem[a] != 0])
            if rng.random() < 0.7:
                pos = (pos + 4) % P
                a_r = pos
            else:
                a_r = int(rng.integers(0, P))
            a_w = a_r if rng.random() < 0.5 else int(rng.integers(0, P))
            if hr[j]:
                ra[j] = a_r
                rv[j] = mem[a_r]
            if hw[j]:
                wa[j] = a_w
                inc[j] = (int(wv[j]) - int(mem[a_w])) % Q
                mem[a_w] = int(wv[j])
        for b in range(te):
            cols.append((ra >> b) & 1)
        for b in range(te):
            cols.append((wa >> b) & 1)
        cols += [hr, hw, wv, rv, inc]
        twist.append(dict(ell_addr=te, k=P, d=1, n_side=P, ell=te, init=init))
    bus = np.array([[int(v) % Q for v in c] for c in cols], dtype=np.uint64)
    buses = [np.ascontiguousarray(bus[:, c * steps:(c + 1) * steps]) for c in range(n_chunks)]
    return buses, dict(steps=steps, shout=shout, twist=twist), inits


def trace_events(z: np.ndarray, mem: dict, m: int):
    """The memory events a witness's shared-CPU-bus tail encodes, in the form
    neo_gpu_shard_fold_step_trace takes: (bus_base, shout, twist) with
    shout[i] = (has_lookup, key, val) and twist[i] = (has_read, ra, rv,
    has_write, wa, wv) per trace step (column order of the bus: per Shout
    [addr bits, has_lookup, val], per Twist [ra bits, wa bits, has_read,
    has_write, wv, rv, inc])."""
    steps = mem["steps"]
    widths = [sd["ell_addr"] + 2 for sd in mem["shout"]] + [2 * td["ell_addr"] + 5 for td in mem["twist"]]
    base = m - sum(widths) * steps
    bus = np.asarray(z, np.uint64)[base:].reshape(sum(widths), steps)

    def bits(rows):
        out = np.zeros(steps, np.uint64)
        for b in range(rows.shape[0]):
            out |= rows[b].astype(np.uint64) << np.uint64(b)
        return out

    shout, twist, col = [], [], 0
    for sd in mem["shout"]:
        e = sd["ell_addr"]
        shout.append((bus[col + e].astype(np.uint8), bits(bus[col:col + e]), bus[col + e + 1].copy()))
        col += e + 2
    for td in mem["twist"]:
        e = td["ell_addr"]
        t = bus[col:col + 2 * e + 5]
        twist.append((t[2 * e].astype(np.uint8), bits(t[:e]), t[2 * e + 3].copy(), t[2 * e + 1].astype(np.uint8),
                      bits(t[e:2 * e]), t[2 * e + 2].copy()))
        col += 2 * e + 5
    return base, shout, twist


def make_memory_workload(ell: int, seed: int, steps: int, shout_ell, twist_ell, m_in: int = 1,
                         table_len: int = None, **trace_kw):
    """Single shard with memory: a satisfied R1CS of n = m = 2^ell whose witness
    carries the shared CPU bus (the Twist / Shout columns of `steps` trace steps)
    in its tail, bus cell (col, j) at m - bus_cols*steps + col*steps + j."""
    m = 1 << ell
    bus, mem = memory_trace(steps, shout_ell, twist_ell, seed + 1, table_len, **trace_kw)
    rng = np.random.default_rng(seed + 2)
    z = rng.integers(0, 1 << 32, size=m, dtype=np.uint64)
    z[0] = 1
    base = m - bus.shape[0] * steps
    if base < m_in or m_in + steps > m:
        raise ValueError("bus does not fit the witness")
    z[base:] = bus.reshape(-1)
    ccs, z = make_r1cs(ell, seed, z=z)
    return ccs, z, mem


def make_memory_workload_chunks(ell: int, seed: int, n_chunks: int, steps: int, shout_ell, twist_ell, m_in: int = 1,
                                table_len: int = None, **trace_kw):
    """A shard whose fold steps prove consecutive chunks of one trace: a
    satisfied R1CS of n = m = 2^ell whose constraints avoid the bus region, and
    per chunk a witness carrying that chunk's bus columns in its tail.
    Returns (ccs, [z per chunk], mem, [Twist MemInits per chunk])."""
    m = 1 << ell
    buses, mem, inits = memory_trace_chunks(n_chunks, steps, shout_ell, twist_ell, seed + 1, table_len, **trace_kw)
    rng = np.random.default_rng(seed + 2)
    z = rng.integers(0, 1 << 32, size=m, dtype=np.uint64)
    z[0] = 1
    base = m - buses[0].shape[0] * steps
    if base < m_in + 4 or m_in + steps > m:
        raise ValueError("bus does not fit the witness")
    ccs, z = make_r1cs(ell, seed, z=z, max_col=base)
    zs = []
    for bus in buses:
        zc = z.copy()
        zc[base:] = bus.reshape(-1)
        zs.append(zc)
    return ccs, zs, mem, inits
