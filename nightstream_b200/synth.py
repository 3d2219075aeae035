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


def make_r1cs(ell: int, seed: int, z_bits: int = 32):
    """Return (ccs, z) for a satisfied random R1CS with n = m = 2^ell."""
    n = m = 1 << ell
    rng = np.random.default_rng(seed)
    z = rng.integers(0, 1 << z_bits, size=m, dtype=np.uint64)
    z[0] = 1
    a_cols = _distinct_cols(rng, n, m, 3)
    b_cols = _distinct_cols(rng, n, m, 3)
    c_cols = _distinct_cols(rng, n, m, 3)
    # the solved column must hold a nonzero witness value
    zero = z[c_cols[:, 2]] == 0
    while zero.any():
        c_cols[zero, 2] = rng.integers(0, m, size=int(zero.sum()))
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
