"""ctypes bindings of the CPU restatement (``libneo_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py, as the checker.  The product never imports
this package.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libneo_oracle.so")
_lib = None

P = ctypes.c_void_p
I = ctypes.c_int
I64 = ctypes.c_int64
SZ = ctypes.c_size_t


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        sigs = {
            "or_fq_mul_batch": [P, P, SZ, P],
            "or_k_mul_batch": [P, P, SZ, P],
            "or_k_inv_batch": [P, SZ, P],
            "or_rq_mul": [P, P, P],
            "or_commit_digits": [P, I, I64, P, P, I],
            "or_commit_fq": [P, I, I64, P, P],
            "or_decomp_b2": [P, I64, P],
            "or_recompose_b2": [P, I64, P],
            "or_rlc_mix": [P, P, I, I64, P, I],
            "or_split_b": [P, I64, I, I, P, P],
            "or_rot_matrix": [P, P],
            "or_interpolate": [P, P, I, P],
            "or_poly_eval_k": [P, I, P, P],
            "or_chi_table": [P, I, P],
            "or_ccs_oracle_new": [P, P, I, I, P, P, P, P, P, I, I, I],
            "or_ccs_oracle_free": [P],
            "or_ccs_oracle_num_rounds": [P],
            "or_ccs_oracle_evals": [P, P, I, P],
            "or_ccs_oracle_fold": [P, P],
            "or_ccs_oracle_me_outputs": [P, P, P],
            "or_ccs_sumcheck_fixed": [P, P, P, P, P],
            "or_q_sum_hypercube": [P, P, I, I, P, P, P, P, P, I, I, P],
            "or_q_eval_ext": [P, P, I, I, P, P, P, P, P, I, I, P, P, P],
            "or_me_y_at_r": [P, P, I, P, I, P, P],
            "or_poseidon2_permute": [P],
            "or_poseidon2_w16_permute": [P],
            "or_chacha8_sample": [P, ctypes.c_uint32, P, ctypes.c_uint64, P],
            "or_pp_setup": [P, ctypes.c_uint32, ctypes.c_uint64, I, P],
            "or_ccs_digest": [P, P],
            "or_tr_new": [ctypes.c_char_p],
            "or_tr_free": [P],
            "or_tr_clone": [P],
            "or_tr_append_message": [P, ctypes.c_char_p, P, SZ],
            "or_tr_append_fields": [P, ctypes.c_char_p, P, SZ],
            "or_tr_append_u64s": [P, ctypes.c_char_p, P, SZ],
            "or_tr_challenge_field": [P, ctypes.c_char_p],
            "or_tr_challenge_fields": [P, ctypes.c_char_p, SZ, P],
            "or_tr_digest32": [P, P],
            "or_tr_state": [P, P],
            "or_mem_oracle_new": [I, I, P, I, P, P, I, P, P, P],
            "or_mem_oracle_free": [P],
            "or_mem_oracle_num_rounds": [P],
            "or_mem_oracle_degree_bound": [P],
            "or_mem_oracle_evals": [P, P, I, P],
            "or_mem_oracle_fold": [P, P],
            "or_addr_lookup_weights": [I, P, I, P, P, P, SZ, P, P],
            "or_twist_addr_new": [I, I, P, I, SZ, P, P, P],
            "or_twist_addr_free": [P],
            "or_twist_addr_num_rounds": [P],
            "or_twist_addr_evals": [P, P, I, P],
            "or_twist_addr_fold": [P, P],
            "or_bus_openings": [P, I64, I64, I64, I, I64, P, I, P, P],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = I if name in ("or_split_b", "or_ccs_oracle_num_rounds", "or_ccs_sumcheck_fixed",
                                        "or_mem_oracle_num_rounds", "or_mem_oracle_degree_bound",
                                        "or_twist_addr_num_rounds") else None
        L.or_ccs_oracle_new.restype = P
        L.or_mem_oracle_new.restype = P
        L.or_twist_addr_new.restype = P
        L.or_tr_new.restype = P
        L.or_tr_clone.restype = P
        L.or_tr_challenge_field.restype = ctypes.c_uint64
        _lib = L
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data


def u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def fq_mul(a, b):
    a, b = u64(a), u64(b)
    out = np.empty_like(a)
    lib().or_fq_mul_batch(ptr(a), ptr(b), a.size, ptr(out))
    return out


def k_mul(a, b):
    a, b = u64(a), u64(b)
    out = np.empty_like(a)
    lib().or_k_mul_batch(ptr(a), ptr(b), a.size // 2, ptr(out))
    return out


def rq_mul(a, b):
    a, b = u64(a), u64(b)
    out = np.empty(54, np.uint64)
    lib().or_rq_mul(ptr(a), ptr(b), ptr(out))
    return out


def commit_digits(pp, Z, threads=0):
    """pp [kappa][m][54] uint64, Z [54][m] int8 -> [kappa][54]"""
    pp = u64(pp)
    Z = np.ascontiguousarray(Z, dtype=np.int8)
    kappa, m = pp.shape[0], pp.shape[1]
    out = np.empty((kappa, 54), np.uint64)
    lib().or_commit_digits(ptr(pp), kappa, m, ptr(Z), ptr(out), threads)
    return out


def commit_fq(pp, Z):
    pp, Z = u64(pp), u64(Z)
    kappa, m = pp.shape[0], pp.shape[1]
    out = np.empty((kappa, 54), np.uint64)
    lib().or_commit_fq(ptr(pp), kappa, m, ptr(Z), ptr(out))
    return out


def decomp_b2(z):
    z = u64(z)
    Z = np.empty((54, z.size), np.int8)
    lib().or_decomp_b2(ptr(z), z.size, ptr(Z))
    return Z


def recompose_b2(Z):
    Z = np.ascontiguousarray(Z, dtype=np.int8)
    z = np.empty(Z.shape[1], np.uint64)
    lib().or_recompose_b2(ptr(Z), Z.shape[1], ptr(z))
    return z


def rlc_mix(rho_coeffs, Zs, threads=0):
    rho = np.ascontiguousarray(rho_coeffs, dtype=np.int8)
    Zs = np.ascontiguousarray(Zs, dtype=np.int8)
    count, _, m = Zs.shape
    out = np.empty((54, m), np.int32)
    lib().or_rlc_mix(ptr(rho), ptr(Zs), count, m, ptr(out), threads)
    return out


def split_b(Zmix, k=12, b=2):
    Zmix = np.ascontiguousarray(Zmix, dtype=np.int32)
    planes = np.empty((k,) + Zmix.shape, np.int8)
    nz = np.empty(k, np.uint8)
    rc = lib().or_split_b(ptr(Zmix), Zmix.size, k, b, ptr(planes), ptr(nz))
    if rc != 0:
        raise ValueError("DEC split: value out of range for k_rho digits")
    return planes, nz.astype(bool)


def rot_matrix(a):
    a = np.ascontiguousarray(a, dtype=np.int8)
    out = np.empty((54, 54), np.uint64)
    lib().or_rot_matrix(ptr(a), ptr(out))
    return out


def interpolate(xs, ys):
    xs, ys = u64(xs), u64(ys)
    out = np.empty_like(ys)
    lib().or_interpolate(ptr(xs), ptr(ys), xs.shape[0], ptr(out))
    return out


def poly_eval_k(coeffs, x):
    coeffs, x = u64(coeffs), u64(x)
    out = np.empty(2, np.uint64)
    lib().or_poly_eval_k(ptr(coeffs), coeffs.shape[0], ptr(x), ptr(out))
    return out


def chi_table(bits):
    bits = u64(bits)
    out = np.empty((1 << bits.shape[0], 2), np.uint64)
    lib().or_chi_table(ptr(bits), bits.shape[0], ptr(out))
    return out


class CcsOracle:
    """Pi_CCS optimized oracle restatement (RoundOracle: evals_at / fold)."""

    def __init__(self, ccs, Z, b, alpha, beta_a, beta_r, gamma, r_inputs, ell_d, ell_n, d_sc):
        self.ccs = ccs
        self.desc = ccs.desc()
        self.Z = np.ascontiguousarray(Z, dtype=np.int8)
        self.k = self.Z.shape[0]
        self._ch = [u64(alpha), u64(beta_a), u64(beta_r), u64(gamma),
                    None if r_inputs is None else u64(r_inputs)]
        self.ell_d, self.ell_n, self.d_sc = ell_d, ell_n, d_sc
        self.h = lib().or_ccs_oracle_new(ctypes.byref(self.desc), ptr(self.Z), self.k, b,
                                         *[ptr(c) for c in self._ch], ell_d, ell_n, d_sc)
        if not self.h:
            raise ValueError("oracle construction failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_ccs_oracle_free(self.h)
            self.h = None

    def num_rounds(self):
        return self.ell_n + self.ell_d

    def evals_at(self, xs):
        xs = u64(xs)
        ys = np.empty_like(xs)
        lib().or_ccs_oracle_evals(self.h, ptr(xs), xs.shape[0], ptr(ys))
        return ys

    def fold(self, r):
        r = u64(r)
        lib().or_ccs_oracle_fold(self.h, ptr(r))

    def me_outputs(self):
        t = self.ccs.t
        y = np.empty((self.k, t, 54, 2), np.uint64)
        ys = np.empty((self.k, t, 2), np.uint64)
        lib().or_ccs_oracle_me_outputs(self.h, ptr(y), ptr(ys))
        return y, ys

    def sumcheck_fixed(self, initial_sum, chals):
        rounds = self.num_rounds()
        ev = np.empty((rounds, self.d_sc + 1, 2), np.uint64)
        fin = np.empty(2, np.uint64)
        rc = lib().or_ccs_sumcheck_fixed(self.h, ptr(u64(initial_sum)), ptr(u64(chals)), ptr(ev), ptr(fin))
        return rc, ev, fin


def q_sum_hypercube(ccs, Z, b, alpha, beta_a, beta_r, gamma, r_inputs, ell_d, ell_n):
    desc = ccs.desc()
    Z = np.ascontiguousarray(Z, dtype=np.int8)
    out = np.empty(2, np.uint64)
    lib().or_q_sum_hypercube(ctypes.byref(desc), ptr(Z), Z.shape[0], b, ptr(u64(alpha)), ptr(u64(beta_a)),
                             ptr(u64(beta_r)), ptr(u64(gamma)),
                             None if r_inputs is None else ptr(u64(r_inputs)), ell_d, ell_n, ptr(out))
    return out


def q_eval_ext(ccs, Z, b, alpha, beta_a, beta_r, gamma, r_inputs, ell_d, ell_n, alpha_p, r_p):
    desc = ccs.desc()
    Z = np.ascontiguousarray(Z, dtype=np.int8)
    out = np.empty(2, np.uint64)
    ri = None if r_inputs is None else u64(r_inputs)
    lib().or_q_eval_ext(ctypes.byref(desc), ptr(Z), Z.shape[0], b, ptr(u64(alpha)), ptr(u64(beta_a)),
                        ptr(u64(beta_r)), ptr(u64(gamma)), ptr(ri), ell_d, ell_n,
                        ptr(u64(alpha_p)), ptr(u64(r_p)), ptr(out))
    return out


def me_y_at_r(ccs, Z, ell_n, r, b=2):
    desc = ccs.desc()
    Z = np.ascontiguousarray(Z, dtype=np.int8)
    y = np.empty((ccs.t, 54, 2), np.uint64)
    ys = np.empty((ccs.t, 2), np.uint64)
    lib().or_me_y_at_r(ctypes.byref(desc), ptr(Z), ell_n, ptr(u64(r)), b, ptr(y), ptr(ys))
    return y, ys


class Transcript:
    """Poseidon2 sponge transcript restatement (neo-transcript/src/poseidon2.rs)."""

    def __init__(self, app_label: bytes):
        self.h = lib().or_tr_new(app_label)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_tr_free(self.h)
            self.h = None

    def clone_state(self):
        """A copy of the sponge (the reference's Clone, used by fork())."""
        c = Transcript.__new__(Transcript)
        c.h = lib().or_tr_clone(self.h)
        return c

    def append_message(self, label: bytes, msg: bytes = b""):
        buf = np.frombuffer(msg, dtype=np.uint8) if msg else np.zeros(1, np.uint8)
        lib().or_tr_append_message(self.h, label, buf.ctypes.data, len(msg))

    def append_fields(self, label: bytes, fs):
        fs = np.ascontiguousarray(np.asarray(fs, dtype=np.uint64).reshape(-1))
        lib().or_tr_append_fields(self.h, label, fs.ctypes.data if fs.size else None, fs.size)

    def append_u64s(self, label: bytes, us):
        us = u64(us)
        lib().or_tr_append_u64s(self.h, label, us.ctypes.data, us.size)

    def challenge_field(self, label: bytes) -> int:
        return int(lib().or_tr_challenge_field(self.h, label))

    def challenge_fields(self, label: bytes, n: int):
        out = np.empty(n, np.uint64)
        lib().or_tr_challenge_fields(self.h, label, n, out.ctypes.data)
        return out

    def digest32(self) -> bytes:
        out = np.empty(32, np.uint8)
        lib().or_tr_digest32(self.h, out.ctypes.data)
        return out.tobytes()

    def state(self):
        out = np.empty(8, np.uint64)
        lib().or_tr_state(self.h, out.ctypes.data)
        return out


def chacha8_sample(seeds, counts, bound):
    """Per stream (32-byte ChaCha8 seed) the first counts[s] next_u64() values
    < bound (sample_uniform_fq for bound = q, crates/neo-ajtai/src/commit.rs:21-30)."""
    seeds = np.ascontiguousarray(np.frombuffer(b"".join(seeds), np.uint8))
    counts = u64(counts)
    out = np.empty(int(counts.sum()), np.uint64)
    lib().or_chacha8_sample(ptr(seeds), len(counts), ptr(counts), int(bound), ptr(out))
    return out


def pp_setup(seed: bytes, kappa: int, m: int, mode: int):
    """Ajtai setup (mode 0, commit.rs:133-157) / setup_par (mode 1, commit.rs:159-225)
    with ChaCha8Rng::from_seed(seed): PP as uint64 [kappa][m][54]."""
    assert len(seed) == 32
    sb = np.frombuffer(seed, np.uint8).copy()
    out = np.empty((kappa, m, 54), np.uint64)
    lib().or_pp_setup(ptr(sb), kappa, m, mode, ptr(out))
    return out


def ccs_digest(ccs):
    desc = ccs.desc()
    out = np.empty(4, np.uint64)
    lib().or_ccs_digest(ctypes.byref(desc), out.ctypes.data)
    return out


MEM_SHOUT_VALUE, MEM_SHOUT_ADAPTER, MEM_BITNESS, MEM_TWIST_READ, MEM_TWIST_WRITE, MEM_VAL_EVAL, MEM_TOTAL_INC, \
    MEM_PRODUCT = range(8)


class MemOracle:
    """Twist / Shout time-lane oracle restatement (literal sparse algorithm of
    crates/neo-memory/src/twist_oracle.rs). cols: uint64 [n_cols, 2^ell, 2]."""

    def __init__(self, kind, cols, r_point=None, r_addr=None, init=None, weights=None):
        self.cols = u64(cols)
        n_cols, L = self.cols.shape[0], self.cols.shape[1]
        ell = L.bit_length() - 1
        ell_addr = 0 if r_addr is None else len(r_addr)
        self._keep = [None if r_point is None else u64(r_point), None if r_addr is None else u64(r_addr),
                      None if init is None else u64(init), None if weights is None else u64(weights)]
        self.claim = np.zeros(2, np.uint64)
        self.h = lib().or_mem_oracle_new(kind, ell, ptr(self._keep[0]), ell_addr, ptr(self._keep[1]),
                                         ptr(self._keep[2]), n_cols, ptr(self.cols), ptr(self._keep[3]),
                                         ptr(self.claim))
        if not self.h:
            raise ValueError("memory oracle construction failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_mem_oracle_free(self.h)
            self.h = None

    def num_rounds(self):
        return lib().or_mem_oracle_num_rounds(self.h)

    def degree_bound(self):
        return lib().or_mem_oracle_degree_bound(self.h)

    def evals_at(self, xs):
        xs = u64(xs)
        ys = np.empty_like(xs)
        lib().or_mem_oracle_evals(self.h, ptr(xs), xs.shape[0], ptr(ys))
        return ys

    def fold(self, r):
        lib().or_mem_oracle_fold(self.h, ptr(u64(r)))


def addr_lookup_weights(r_cycle, has_lookup, addr_bits, table):
    """AddressLookupOracle weight table and claimed sum (twist_oracle.rs:1671-1724)."""
    r_cycle, has_lookup, addr_bits, table = u64(r_cycle), u64(has_lookup), u64(addr_bits), u64(table)
    ell, ell_addr = r_cycle.shape[0], addr_bits.shape[0]
    w = np.empty((1 << ell_addr, 2), np.uint64)
    claim = np.empty(2, np.uint64)
    lib().or_addr_lookup_weights(ell, ptr(r_cycle), ell_addr, ptr(has_lookup), ptr(addr_bits), ptr(table),
                                 table.shape[0], ptr(w), ptr(claim))
    return w, claim


class TwistAddrOracle:
    """Twist address-lane read (kind 0) / write (kind 1) check oracle
    (twist_oracle.rs:1259-1642); degree bound 2, ell_addr rounds."""

    def __init__(self, kind, cols, r_cycle, ell_addr, init_pairs=()):
        self.cols = u64(cols)
        L = self.cols.shape[1]
        ell = L.bit_length() - 1
        self._r = u64(r_cycle)
        ia = np.array([a for a, _ in init_pairs], np.uint64) if init_pairs else np.zeros(1, np.uint64)
        iv = u64(np.array([v for _, v in init_pairs], np.uint64).reshape(-1, 2)) if init_pairs else np.zeros((1, 2), np.uint64)
        self._init = (ia, iv)
        self.h = lib().or_twist_addr_new(kind, ell, ptr(self._r), ell_addr, len(init_pairs), ptr(ia), ptr(iv),
                                         ptr(self.cols))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_twist_addr_free(self.h)
            self.h = None

    def num_rounds(self):
        return lib().or_twist_addr_num_rounds(self.h)

    def degree_bound(self):
        return 2

    def evals_at(self, xs):
        xs = u64(xs)
        ys = np.empty_like(xs)
        lib().or_twist_addr_evals(self.h, ptr(xs), xs.shape[0], ptr(ys))
        return ys

    def fold(self, r):
        lib().or_twist_addr_fold(self.h, ptr(u64(r)))


def bus_openings(Z, bus_base, chunk, n_cols, m_in, r):
    """Bus-column openings of a digit witness at r (cpu_bus.rs:195-320)."""
    Z = np.ascontiguousarray(Z, np.int8)
    r = u64(r)
    y = np.empty((n_cols, 54, 2), np.uint64)
    ysc = np.empty((n_cols, 2), np.uint64)
    lib().or_bus_openings(ptr(Z), Z.shape[1], bus_base, chunk, n_cols, m_in, ptr(r), r.shape[0], ptr(y), ptr(ysc))
    return y, ysc
