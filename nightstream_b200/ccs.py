"""CCS structure on the host, in the layout the C-ABI takes.

Mirrors ``CcsStructure { matrices: Vec<CcsMatrix>, f: SparsePoly, n, m }``
(crates/neo-ccs/src/relations.rs:14-23) with each matrix either the identity
sentinel or CSC (crates/neo-ccs/src/sparse.rs:19, 151-191), and
``r1cs_to_ccs`` (crates/neo-ccs/src/r1cs.rs:13-43): for square R1CS the CCS is
identity-first, matrices [I, A, B, C] and f = X1*X2 - X3.
"""
import ctypes
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from .params import Q


class CcsDesc(ctypes.Structure):
    """C view of a CCS (``neo_ccs_desc`` in include/neo_gpu.h)."""
    _fields_ = [
        ("n", ctypes.c_uint32),
        ("m", ctypes.c_uint32),
        ("t", ctypes.c_uint32),
        ("is_identity", ctypes.c_void_p),
        ("col_ptr", ctypes.c_void_p),
        ("nnz_off", ctypes.c_void_p),
        ("row_idx", ctypes.c_void_p),
        ("vals", ctypes.c_void_p),
        ("n_terms", ctypes.c_uint32),
        ("f_coeff", ctypes.c_void_p),
        ("f_exps", ctypes.c_void_p),
    ]


@dataclass
class CscMatrix:
    n: int
    m: int
    col_ptr: np.ndarray  # int64/uint64 [m+1]
    row_idx: np.ndarray  # uint32 [nnz]
    vals: np.ndarray     # uint64 [nnz], canonical

    @property
    def nnz(self) -> int:
        return int(self.row_idx.shape[0])

    @staticmethod
    def from_coo(n: int, m: int, rows, cols, vals) -> "CscMatrix":
        rows = np.asarray(rows, dtype=np.int64)
        cols = np.asarray(cols, dtype=np.int64)
        vals = np.asarray(vals, dtype=np.uint64)
        order = np.lexsort((rows, cols))
        rows, cols, vals = rows[order], cols[order], vals[order]
        counts = np.bincount(cols, minlength=m)
        col_ptr = np.zeros(m + 1, dtype=np.uint64)
        col_ptr[1:] = np.cumsum(counts).astype(np.uint64)
        return CscMatrix(n, m, col_ptr, rows.astype(np.uint32), vals)

    def to_csr(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        cols = np.repeat(np.arange(self.m, dtype=np.uint32),
                         np.diff(self.col_ptr.astype(np.int64)))
        order = np.lexsort((cols, self.row_idx))
        r, c, v = self.row_idx[order], cols[order], self.vals[order]
        counts = np.bincount(r.astype(np.int64), minlength=self.n)
        row_ptr = np.zeros(self.n + 1, dtype=np.uint64)
        row_ptr[1:] = np.cumsum(counts).astype(np.uint64)
        return row_ptr, c.astype(np.uint32), v


@dataclass
class CcsStructure:
    n: int
    m: int
    matrices: List[Optional[CscMatrix]]          # None = identity sentinel
    f_terms: List[Tuple[int, List[int]]]         # (coeff mod q, exps[t])

    @property
    def t(self) -> int:
        return len(self.matrices)

    @property
    def f_degree(self) -> int:
        return max(sum(e) for _, e in self.f_terms)

    def desc(self) -> CcsDesc:
        """Flatten into the C struct; arrays are kept alive by this object."""
        t, m = self.t, self.m
        is_id = np.array([1 if M is None else 0 for M in self.matrices], dtype=np.uint8)
        col_ptr = np.zeros((t, m + 1), dtype=np.uint64)
        nnz_off = np.zeros(t + 1, dtype=np.uint64)
        rows, vals = [], []
        for j, M in enumerate(self.matrices):
            if M is not None:
                col_ptr[j] = M.col_ptr
                rows.append(M.row_idx)
                vals.append(M.vals)
                nnz_off[j + 1] = nnz_off[j] + M.nnz
            else:
                nnz_off[j + 1] = nnz_off[j]
        row_idx = np.ascontiguousarray(np.concatenate(rows) if rows else np.zeros(1, np.uint32), dtype=np.uint32)
        vv = np.ascontiguousarray(np.concatenate(vals) if vals else np.zeros(1, np.uint64), dtype=np.uint64)
        f_coeff = np.array([c % Q for c, _ in self.f_terms], dtype=np.uint64)
        f_exps = np.array([e for _, e in self.f_terms], dtype=np.uint32).reshape(-1)
        keep = [is_id, col_ptr, nnz_off, row_idx, vv, f_coeff, f_exps]
        d = CcsDesc()
        d._keep = keep  # the struct owns the arrays it points to
        d.n, d.m, d.t = self.n, self.m, t
        d.is_identity = is_id.ctypes.data
        d.col_ptr = col_ptr.ctypes.data
        d.nnz_off = nnz_off.ctypes.data
        d.row_idx = row_idx.ctypes.data
        d.vals = vv.ctypes.data
        d.n_terms = len(self.f_terms)
        d.f_coeff = f_coeff.ctypes.data
        d.f_exps = f_exps.ctypes.data
        return d


def r1cs_to_ccs(n: int, m: int, A: CscMatrix, B: CscMatrix, C: CscMatrix) -> CcsStructure:
    """Identity-first CCS for square R1CS (crates/neo-ccs/src/r1cs.rs:13-43)."""
    if n == m:
        return CcsStructure(n, m, [None, A, B, C],
                            [(1, [0, 1, 1, 0]), (Q - 1, [0, 0, 0, 1])])
    return CcsStructure(n, m, [A, B, C], [(1, [1, 1, 0]), (Q - 1, [0, 0, 1])])
