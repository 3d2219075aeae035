"""ctypes binding of libneo_gpu.so (include/neo_gpu.h).

Every call goes through the C ABI with host buffers, exactly as a Rust or C
caller would bind it.  There is no CPU fallback: if the CUDA library is
missing or no GPU is present, loading fails with an exception.
"""
import ctypes
import os

import numpy as np

from .ccs import CcsDesc

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libneo_gpu.so")

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I = ctypes.c_int

NEO_OK = 0
_ERRS = {1: "NEO_ERR_ARG", 2: "NEO_ERR_OOM", 3: "NEO_ERR_INVARIANT", 4: "NEO_ERR_CUDA", 5: "NEO_ERR_UNSUPPORTED",
         6: "NEO_ERR_CANCELLED"}

# symbol -> argtypes; every function returns int unless listed in _RESTYPES
SIGNATURES = {
    "neo_gpu_ctx_create": [I, P],
    "neo_gpu_ctx_destroy": [P],
    "neo_gpu_last_error": [P],
    "neo_gpu_kernel_launches": [P],
    "neo_gpu_pp_upload": [P, U32, U64, P],
    "neo_gpu_pp_generate": [P, P, U32, U64, I],
    "neo_gpu_pp_download": [P, U64, U64, U64, P],
    "neo_gpu_chacha8_sample": [P, P, U32, P, U64, P],
    "neo_gpu_commit": [P, P, U32, U64, P],
    "neo_gpu_decomp_b2": [P, P, U64, P],
    "neo_gpu_rlc_mix": [P, P, P, U32, U64, P],
    "neo_gpu_split_b": [P, P, U64, U32, U32, P, P],
    "neo_gpu_me_y": [P, P, P, U32, U32, P, U32, P, P],
    "neo_gpu_ccs_oracle_create": [P, P, P, U32, U32, P, P, P, P, P, U32, U32, U32, P],
    "neo_gpu_ccs_oracle_evals": [P, P, U32, P],
    "neo_gpu_ccs_oracle_fold": [P, P],
    "neo_gpu_ccs_oracle_num_rounds": [P],
    "neo_gpu_ccs_oracle_row_rounds_device": [P, P, U32, ctypes.c_void_p],
    "neo_gpu_ccs_oracle_degree_bound": [P],
    "neo_gpu_ccs_oracle_me_outputs": [P, P, P],
    "neo_gpu_ccs_oracle_destroy": [P],
    "neo_gpu_ctx_stream": [P, P],
    "neo_gpu_synchronize": [P],
    "neo_gpu_commit_device": [P, ctypes.c_void_p, U32, U64, ctypes.c_void_p],
    "neo_gpu_commit_device_ex": [P, ctypes.c_void_p, U32, U64, ctypes.c_void_p, U32],
    "neo_gpu_commit_noalloc": [P, ctypes.c_void_p, U32, U64, ctypes.c_void_p],
    "neo_gpu_mix_rhos_commits": [P, P, P, U32, U32, P],
    "neo_gpu_shard_step_proof": [P, P, U64, P],
    "neo_gpu_ccs_autotune": [P, P, P, U32, U32, P],
    "neo_gpu_tune_load": [ctypes.c_char_p],
    "neo_gpu_tune_save": [ctypes.c_char_p],
    "neo_gpu_tune_get": [U32, U32, P],
    "neo_gpu_combine_b_pows": [P, P, U32, U32, U32, P],
    "neo_gpu_shard_step_stats": [P, P, U32],
    "neo_gpu_shard_create": [P, P, U32, U32, ctypes.c_char_p, P],
    "neo_gpu_shard_create_mem": [P, P, U32, U32, ctypes.c_char_p, P, P],
    "neo_gpu_shard_val_obligations": [P, P],
    "neo_gpu_shard_checkpoint": [P, P, U64, P],
    "neo_gpu_shard_restore": [P, P, U64],
    "neo_gpu_shard_set_twist_init": [P, U32, U64, P, P],
    "neo_gpu_shard_fold_step": [P, P, P, U64, P],
    "neo_gpu_shard_fold_step_device": [P, ctypes.c_void_p, P],
    "neo_gpu_shard_fold_step_trace": [P, P, U64, P, P, U64, P],
    "neo_gpu_shard_transcript_state": [P, P],
    "neo_gpu_shard_ccs_digest": [P, P],
    "neo_gpu_shard_destroy": [P],
    "neo_gpu_batch_create": [I, U32, P],
    "neo_gpu_batch_set_reserve": [P, U64],
    "neo_gpu_batch_submit": [P, P, P, U32, U32, U32, ctypes.c_char_p, P],
    "neo_gpu_batch_wait_all": [P, ctypes.c_double],
    "neo_gpu_batch_submit_chunks": [P, P, P, P, P, U32, U32, U32, ctypes.c_char_p, P],
    "neo_gpu_batch_submit_mem": [P, P, P, P, U32, U32, U32, ctypes.c_char_p, P],
    "neo_gpu_batch_job_info": [P, U64, P, P, P],
    "neo_gpu_batch_job_error": [P, U64, P, U64],
    "neo_gpu_batch_cancel": [P, U64],
    "neo_gpu_wait_probe": [P, U32, U32],
    "neo_gpu_batch_kernel_launches": [P],
    "neo_gpu_batch_destroy": [P],
    "neo_transcript_new": [ctypes.c_char_p, P],
    "neo_transcript_append_message": [P, ctypes.c_char_p, P, ctypes.c_size_t],
    "neo_transcript_append_fields": [P, ctypes.c_char_p, P, ctypes.c_size_t],
    "neo_transcript_append_u64s": [P, ctypes.c_char_p, P, ctypes.c_size_t],
    "neo_transcript_challenge_field": [P, ctypes.c_char_p, P],
    "neo_transcript_challenge_fields": [P, ctypes.c_char_p, ctypes.c_size_t, P],
    "neo_transcript_digest32": [P, P],
    "neo_transcript_state": [P, P],
    "neo_transcript_destroy": [P],
    "neo_ccs_digest": [P, P],
    "neo_gpu_mem_oracle_create": [P, I, U32, P, U32, P, P, U32, P, P, P, P],
    "neo_gpu_mem_oracle_create_device": [P, I, U32, P, U32, P, P, U32, ctypes.c_void_p, P, P, P],
    "neo_gpu_mem_oracle_evals": [P, P, U32, P],
    "neo_gpu_mem_oracle_fold": [P, P],
    "neo_gpu_mem_oracle_num_rounds": [P],
    "neo_gpu_mem_oracle_degree_bound": [P],
    "neo_gpu_mem_oracle_destroy": [P],
    "neo_gpu_addr_lookup_weights": [P, U32, P, U32, P, P, P, U64, P, P],
    "neo_gpu_twist_addr_create": [P, I, U32, P, U32, U64, P, P, P, P],
    "neo_gpu_twist_addr_create_device": [P, I, U32, P, U32, U64, P, P, ctypes.c_void_p, P],
    "neo_gpu_twist_addr_evals": [P, P, U32, P],
    "neo_gpu_twist_addr_fold": [P, P],
    "neo_gpu_twist_addr_num_rounds": [P],
    "neo_gpu_twist_addr_degree_bound": [P],
    "neo_gpu_twist_addr_destroy": [P],
}
_RESTYPES = {
    "neo_gpu_last_error": ctypes.c_char_p,
    "neo_gpu_kernel_launches": U64,
    "neo_gpu_ccs_oracle_num_rounds": U32,
    "neo_gpu_ccs_oracle_degree_bound": U32,
    "neo_gpu_batch_kernel_launches": U64,
    "neo_gpu_mem_oracle_num_rounds": U32,
    "neo_gpu_mem_oracle_degree_bound": U32,
    "neo_gpu_twist_addr_num_rounds": U32,
    "neo_gpu_twist_addr_degree_bound": U32,
}

_lib = None


TUNE_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_b200.txt")


def tune_load(path: str = TUNE_FILE) -> bool:
    """Load a launch-shape table (neo_gpu_tune_load); False when the file is absent."""
    if not os.path.exists(path):
        return False
    return load().neo_gpu_tune_load(path.encode()) == 0


def tune_save(path: str):
    if load().neo_gpu_tune_save(path.encode()):
        raise NeoGpuError(1, f"tune_save {path}")


def tune_get(ell_n: int, k: int):
    out = np.zeros(3, np.uint64)
    if load().neo_gpu_tune_get(ell_n, k, _p(out)):
        return None
    return tuple(int(x) for x in out)


class NeoGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERRS.get(code, code)}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"libneo_gpu.so not built ({path}); run nightstream_b200/build.py")
        L = ctypes.CDLL(path)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, I)
        _lib = L
        if os.path.exists(TUNE_FILE):  # the launch-shape table measured on the target GPU (tune.py)
            L.neo_gpu_tune_load(TUNE_FILE.encode())
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _i8(a):
    return np.ascontiguousarray(a, dtype=np.int8)


class Context:
    """One device + one stream (neo_gpu_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.neo_gpu_ctx_create(device, ctypes.byref(h))
        if rc != NEO_OK:
            raise NeoGpuError(rc, f"context creation failed on device {device}")
        self.h = h

    def check(self, rc):
        if rc != NEO_OK:
            raise NeoGpuError(rc, self.lib.neo_gpu_last_error(self.h).decode())

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.neo_gpu_kernel_launches(self.h))

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self.check(self.lib.neo_gpu_ctx_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self):
        self.check(self.lib.neo_gpu_synchronize(self.h))

    def wait_probe(self, set_flag: bool, spin_limit: int = 1000):
        """Bounded device wait on a flag (neo_gpu_wait_probe); raises NeoGpuError
        (NEO_ERR_CUDA) when the wait runs out."""
        self.check(self.lib.neo_gpu_wait_probe(self.h, 1 if set_flag else 0, spin_limit))

    def commit_device(self, d_digits: int, n_vec: int, m: int, d_out: int, small_digits: bool = False):
        """Asynchronous commitment of device digits; small_digits: the caller
        guarantees |digit| <= 63 (NEO_COMMIT_SMALL_DIGITS)."""
        if small_digits:
            self.check(self.lib.neo_gpu_commit_device_ex(self.h, ctypes.c_void_p(d_digits), n_vec, m,
                                                         ctypes.c_void_p(d_out), 1))
        else:
            self.check(self.lib.neo_gpu_commit_device(self.h, ctypes.c_void_p(d_digits), n_vec, m,
                                                      ctypes.c_void_p(d_out)))

    def commit_noalloc(self, d_digits: int, n_vec: int, m: int, d_out: int):
        """Commitment with the library's fixed device scratch (no allocation)."""
        self.check(self.lib.neo_gpu_commit_noalloc(self.h, ctypes.c_void_p(d_digits), n_vec, m, ctypes.c_void_p(d_out)))

    def mix_rhos_commits(self, rhos: np.ndarray, cs: np.ndarray) -> np.ndarray:
        """sum_i rho_i c_i: rhos [count][54][54] F_q, cs [count][kappa][54] -> [kappa][54]
        (CommitMixers::mix_rhos_commits, crates/neo-fold/src/shard.rs:146-153)."""
        rhos, cs = _u64(rhos), _u64(cs)
        count, kappa = cs.shape[0], cs.shape[1]
        out = np.empty((kappa, 54), np.uint64)
        self.check(self.lib.neo_gpu_mix_rhos_commits(self.h, _p(rhos), _p(cs), count, kappa, _p(out)))
        return out

    def combine_b_pows(self, cs: np.ndarray, b: int) -> np.ndarray:
        """sum_i b^i c_i over cs [count][kappa][54] (CommitMixers::combine_b_pows)."""
        cs = _u64(cs)
        count, kappa = cs.shape[0], cs.shape[1]
        out = np.empty((kappa, 54), np.uint64)
        self.check(self.lib.neo_gpu_combine_b_pows(self.h, _p(cs), count, kappa, b, _p(out)))
        return out

    def ccs_autotune(self, ccs, Z: np.ndarray, reps: int = 3):
        """Time every launch choice of the Pi_CCS row rounds on this CCS and the
        digit matrices Z [k][54][m]; the best is recorded for (ell_n, k) and
        returned as (nc_threads, compact_q, hist_items)."""
        Zs = _i8(Z)
        desc = ccs.desc()
        out = np.zeros(3, np.uint64)
        self.check(self.lib.neo_gpu_ccs_autotune(self.h, ctypes.byref(desc), _p(Zs), Zs.shape[0], reps, _p(out)))
        return tuple(int(x) for x in out)

    def close(self):
        if getattr(self, "h", None):
            self.lib.neo_gpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # -- Ajtai -----------------------------------------------------------
    def pp_upload(self, pp: np.ndarray):
        pp = _u64(pp)
        kappa, m, d = pp.shape
        assert d == 54
        self.check(self.lib.neo_gpu_pp_upload(self.h, kappa, m, _p(pp)))
        self.kappa, self.m = kappa, m

    PP_SETUP, PP_SETUP_PAR = 0, 1

    def pp_generate(self, seed: bytes, kappa: int, m: int, mode: int = 1):
        """Generate and register M on the device: mode 0 = setup, 1 = setup_par,
        both from ChaCha8Rng::from_seed(seed)."""
        if len(seed) != 32:
            raise ValueError("seed must be 32 bytes")
        sb = np.frombuffer(bytes(seed), np.uint8).copy()
        self.check(self.lib.neo_gpu_pp_generate(self.h, _p(sb), kappa, m, mode))
        self.kappa, self.m = kappa, m

    def pp_download(self, m: int = None, kappa: int = None, first: int = 0, count: int = None) -> np.ndarray:
        """Words [first, first + count) of the registered PP of this m; the whole
        [kappa][m][54] array by default."""
        m = self.m if m is None else m
        kappa = self.kappa if kappa is None else kappa
        whole = count is None
        if whole:
            count = kappa * m * 54 - first
        out = np.empty(count, np.uint64)
        self.check(self.lib.neo_gpu_pp_download(self.h, m, first, count, _p(out)))
        return out.reshape(kappa, m, 54) if whole and first == 0 else out

    def chacha8_sample(self, seeds, counts, bound: int) -> np.ndarray:
        """Per 32-byte seed, the first counts[s] ChaCha8 next_u64() values < bound."""
        sb = np.frombuffer(b"".join(bytes(x) for x in seeds), np.uint8).copy()
        counts = _u64(counts)
        out = np.empty(int(counts.sum()), np.uint64)
        self.check(self.lib.neo_gpu_chacha8_sample(self.h, _p(sb), len(counts), _p(counts), int(bound), _p(out)))
        return out

    def commit(self, digits: np.ndarray) -> np.ndarray:
        """digits [n_vec][54][m] (or [54][m]) -> commitments [n_vec][kappa][54]."""
        single = digits.ndim == 2
        Z = _i8(digits[None] if single else digits)
        n_vec, _, m = Z.shape
        out = np.empty((n_vec, self.kappa, 54), np.uint64)
        self.check(self.lib.neo_gpu_commit(self.h, _p(Z), n_vec, m, _p(out)))
        return out[0] if single else out

    def decomp_b2(self, z: np.ndarray) -> np.ndarray:
        z = _u64(z)
        Z = np.empty((54, z.size), np.int8)
        self.check(self.lib.neo_gpu_decomp_b2(self.h, _p(z), z.size, _p(Z)))
        return Z

    # -- RLC / DEC -------------------------------------------------------
    def rlc_mix(self, rho_coeffs: np.ndarray, Zs: np.ndarray) -> np.ndarray:
        rho = _i8(rho_coeffs)
        Zs = _i8(Zs)
        count, _, m = Zs.shape
        out = np.empty((54, m), np.int32)
        self.check(self.lib.neo_gpu_rlc_mix(self.h, _p(rho), _p(Zs), count, m, _p(out)))
        return out

    def split_b(self, Zmix: np.ndarray, k: int = 12, b: int = 2):
        Zmix = np.ascontiguousarray(Zmix, dtype=np.int32)
        planes = np.empty((k,) + Zmix.shape, np.int8)
        nz = np.empty(k, np.uint8)
        self.check(self.lib.neo_gpu_split_b(self.h, _p(Zmix), Zmix.size, k, b, _p(planes), _p(nz)))
        return planes, nz.astype(bool)

    def me_y(self, ccs, Z: np.ndarray, r: np.ndarray, b: int = 2):
        single = Z.ndim == 2
        Zs = _i8(Z[None] if single else Z)
        r = _u64(r)
        desc = ccs.desc()
        n_w = Zs.shape[0]
        y = np.empty((n_w, ccs.t, 54, 2), np.uint64)
        ys = np.empty((n_w, ccs.t, 2), np.uint64)
        self.check(self.lib.neo_gpu_me_y(self.h, ctypes.byref(desc), _p(Zs), n_w, r.shape[0], _p(r), b,
                                         _p(y), _p(ys)))
        return (y[0], ys[0]) if single else (y, ys)


class GpuCcsOracle:
    """Pi_CCS RoundOracle on the GPU (OptimizedOracle, oracle.rs:1566-2104)."""

    def __init__(self, ctx: Context, ccs, Z, b, alpha, beta_a, beta_r, gamma, r_inputs, ell_d, ell_n, d_sc):
        self.ctx = ctx
        self.ccs = ccs
        self._desc = ccs.desc()
        Zs = _i8(Z)
        self.k = Zs.shape[0]
        self.t = ccs.t
        self._keep = [_u64(alpha), _u64(beta_a), _u64(beta_r), _u64(gamma),
                      None if r_inputs is None else _u64(r_inputs)]
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.neo_gpu_ccs_oracle_create(ctx.h, ctypes.byref(self._desc), _p(Zs), self.k, b,
                                                    *[_p(x) for x in self._keep], ell_d, ell_n, d_sc,
                                                    ctypes.byref(h)))
        self.h = h

    def num_rounds(self) -> int:
        return int(self.ctx.lib.neo_gpu_ccs_oracle_num_rounds(self.h))

    def degree_bound(self) -> int:
        return int(self.ctx.lib.neo_gpu_ccs_oracle_degree_bound(self.h))

    def evals_at(self, xs: np.ndarray) -> np.ndarray:
        xs = _u64(xs)
        ys = np.empty_like(xs)
        self.ctx.check(self.ctx.lib.neo_gpu_ccs_oracle_evals(self.h, _p(xs), xs.shape[0], _p(ys)))
        return ys

    def fold(self, r: np.ndarray):
        r = _u64(r)
        self.ctx.check(self.ctx.lib.neo_gpu_ccs_oracle_fold(self.h, _p(r)))

    bind = fold

    def row_rounds_device(self, chals: np.ndarray, d_coeffs: int):
        """Next len(chals) row rounds back to back; coefficients to device memory."""
        chals = _u64(chals)
        self.ctx.check(self.ctx.lib.neo_gpu_ccs_oracle_row_rounds_device(self.h, _p(chals), chals.shape[0],
                                                                         d_coeffs))

    def me_outputs(self):
        y = np.empty((self.k, self.t, 54, 2), np.uint64)
        ys = np.empty((self.k, self.t, 2), np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_ccs_oracle_me_outputs(self.h, _p(y), _p(ys)))
        return y, ys

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h is not None:  # a closed context already released the device
                self.ctx.lib.neo_gpu_ccs_oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


MEM_SHOUT_VALUE, MEM_SHOUT_ADAPTER, MEM_BITNESS, MEM_TWIST_READ, MEM_TWIST_WRITE, MEM_VAL_EVAL, MEM_TOTAL_INC, \
    MEM_PRODUCT = range(8)


class GpuMemOracle:
    """Twist / Shout time-lane RoundOracle on the GPU (crates/neo-memory/src/
    twist_oracle.rs).  cols: uint64 [n_cols, 2^ell, 2] in the C ABI's column
    order for `kind`; claim: the hypercube sum."""

    def __init__(self, ctx: Context, kind: int, cols, r_point=None, r_addr=None, init=None, weights=None):
        self.ctx = ctx
        cols = _u64(cols)
        n_cols, L = cols.shape[0], cols.shape[1]
        ell = L.bit_length() - 1
        if L != 1 << ell:
            raise ValueError("column length must be a power of two")
        self._keep = [None if r_point is None else _u64(r_point), None if r_addr is None else _u64(r_addr),
                      None if init is None else _u64(init), None if weights is None else _u64(weights)]
        ell_addr = 0 if r_addr is None else self._keep[1].shape[0]
        self.claim = np.zeros(2, np.uint64)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.neo_gpu_mem_oracle_create(ctx.h, kind, ell, _p(self._keep[0]), ell_addr, _p(self._keep[1]),
                                                    _p(self._keep[2]), n_cols, _p(cols), _p(self._keep[3]),
                                                    _p(self.claim), ctypes.byref(h)))
        self.h = h

    def num_rounds(self) -> int:
        return int(self.ctx.lib.neo_gpu_mem_oracle_num_rounds(self.h))

    def degree_bound(self) -> int:
        return int(self.ctx.lib.neo_gpu_mem_oracle_degree_bound(self.h))

    def evals_at(self, xs: np.ndarray) -> np.ndarray:
        xs = _u64(xs)
        ys = np.empty_like(xs)
        self.ctx.check(self.ctx.lib.neo_gpu_mem_oracle_evals(self.h, _p(xs), xs.shape[0], _p(ys)))
        return ys

    def fold(self, r: np.ndarray):
        self.ctx.check(self.ctx.lib.neo_gpu_mem_oracle_fold(self.h, _p(_u64(r))))

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h is not None:
                self.ctx.lib.neo_gpu_mem_oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class GpuTwistAddrOracle:
    """Twist address-lane read (0) / write (1) check oracle on the GPU
    (twist_oracle.rs:1259-1642)."""

    def __init__(self, ctx: Context, kind: int, cols, r_cycle, ell_addr: int, init_pairs=()):
        self.ctx = ctx
        cols = _u64(cols)
        ell = cols.shape[1].bit_length() - 1
        self._r = _u64(r_cycle)
        ia = np.array([a for a, _ in init_pairs], np.uint64) if init_pairs else np.zeros(1, np.uint64)
        iv = _u64(np.array([v for _, v in init_pairs], np.uint64).reshape(-1, 2)) if init_pairs else \
            np.zeros((1, 2), np.uint64)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.neo_gpu_twist_addr_create(ctx.h, kind, ell, _p(self._r), ell_addr, len(init_pairs), _p(ia),
                                                    _p(iv), _p(cols), ctypes.byref(h)))
        self.h = h

    def num_rounds(self) -> int:
        return int(self.ctx.lib.neo_gpu_twist_addr_num_rounds(self.h))

    def degree_bound(self) -> int:
        return int(self.ctx.lib.neo_gpu_twist_addr_degree_bound(self.h))

    def evals_at(self, xs: np.ndarray) -> np.ndarray:
        xs = _u64(xs)
        ys = np.empty_like(xs)
        self.ctx.check(self.ctx.lib.neo_gpu_twist_addr_evals(self.h, _p(xs), xs.shape[0], _p(ys)))
        return ys

    def fold(self, r: np.ndarray):
        self.ctx.check(self.ctx.lib.neo_gpu_twist_addr_fold(self.h, _p(_u64(r))))

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h is not None:
                self.ctx.lib.neo_gpu_twist_addr_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def addr_lookup_weights(ctx: Context, r_cycle, has_lookup, addr_bits, table):
    """AddressLookupOracle weight table and claimed sum on the GPU (twist_oracle.rs:1671-1724)."""
    r_cycle, has_lookup, addr_bits, table = _u64(r_cycle), _u64(has_lookup), _u64(addr_bits), _u64(table)
    ell, ell_addr = r_cycle.shape[0], addr_bits.shape[0]
    w = np.empty((1 << ell_addr, 2), np.uint64)
    claim = np.empty(2, np.uint64)
    ctx.check(ctx.lib.neo_gpu_addr_lookup_weights(ctx.h, ell, _p(r_cycle), ell_addr, _p(has_lookup), _p(addr_bits),
                                                  _p(table), table.shape[0], _p(w), _p(claim)))
    return w, claim


class MemInstance(ctypes.Structure):
    _fields_ = [("ell_addr", U32), ("k", U64), ("d", U64), ("n_side", U64), ("ell", U64), ("table", P),
                ("table_len", U64), ("n_init", U64), ("init_addr", P), ("init_val", P)]


class MemInit(ctypes.Structure):
    _fields_ = [("n_init", U64), ("addr", P), ("val", P)]


class MemDesc(ctypes.Structure):
    _fields_ = [("steps", U64), ("n_shout", U32), ("shout", P), ("n_twist", U32), ("twist", P)]


def _mem_desc(mem: dict) -> MemDesc:
    keep = []

    def inst(d, table=None, init=()):
        mi = MemInstance()
        mi.ell_addr, mi.k, mi.d, mi.n_side, mi.ell = d["ell_addr"], d["k"], d["d"], d["n_side"], d["ell"]
        if table is not None:
            t = _u64(table)
            keep.append(t)
            mi.table, mi.table_len = _p(t), t.shape[0]
        if init:
            a = np.array([x for x, _ in init], np.uint64)
            v = np.array([y for _, y in init], np.uint64)
            keep.extend([a, v])
            mi.n_init, mi.init_addr, mi.init_val = len(init), _p(a), _p(v)
        return mi

    sh = mem.get("shout", [])
    tw = mem.get("twist", [])
    sa = (MemInstance * max(1, len(sh)))(*[inst(d, table=d["table"]) for d in sh])
    ta = (MemInstance * max(1, len(tw)))(*[inst(d, init=d.get("init", ())) for d in tw])
    md = MemDesc()
    md.steps = mem["steps"]
    md.n_shout, md.shout = len(sh), ctypes.cast(sa, ctypes.c_void_p).value
    md.n_twist, md.twist = len(tw), ctypes.cast(ta, ctypes.c_void_p).value
    md._keep = (keep, sa, ta)
    return md


class _ShoutEvents(ctypes.Structure):
    _fields_ = [("has_lookup", ctypes.c_void_p), ("key", ctypes.c_void_p), ("val", ctypes.c_void_p)]


class _TwistEvents(ctypes.Structure):
    _fields_ = [("has_read", ctypes.c_void_p), ("ra", ctypes.c_void_p), ("rv", ctypes.c_void_p),
                ("has_write", ctypes.c_void_p), ("wa", ctypes.c_void_p), ("wv", ctypes.c_void_p)]


class _TraceChunk(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_uint64), ("shout", ctypes.c_void_p), ("twist", ctypes.c_void_p)]


class Shard:
    """Shard prover with a device-resident accumulator (neo_gpu_shard)."""

    def __init__(self, ctx: Context, ccs, m_in: int = 1, k_rho: int = 12, app_label: bytes = b"neo/shard",
                 mem: dict = None):
        """mem: None, or dict(steps, shout=[dict(ell_addr, k, d, n_side, ell, table)],
        twist=[dict(ell_addr, k, d, n_side, ell, init=[(addr, value)])])."""
        self.ctx = ctx
        self._desc = ccs.desc()
        h = ctypes.c_void_p()
        if mem and (mem.get("shout") or mem.get("twist")):
            self._mem = _mem_desc(mem)
            ctx.check(ctx.lib.neo_gpu_shard_create_mem(ctx.h, ctypes.byref(self._desc), m_in, k_rho, app_label,
                                                       ctypes.byref(self._mem), ctypes.byref(h)))
        else:
            ctx.check(ctx.lib.neo_gpu_shard_create(ctx.h, ctypes.byref(self._desc), m_in, k_rho, app_label,
                                                   ctypes.byref(h)))
        self.h = h
        self._cap = 0

    def fold_step(self, z: np.ndarray) -> np.ndarray:
        """One fold step; returns the canonical step-proof words."""
        z = _u64(z)
        n = ctypes.c_uint64()
        if self._cap == 0:
            self._cap = 1 << 20
        out = np.empty(self._cap, np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_fold_step(self.h, _p(z), _p(out), self._cap, ctypes.byref(n)))
        return out[: n.value].copy()

    def fold_step_trace(self, z_cpu: np.ndarray, shout=(), twist=()) -> np.ndarray:
        """One fold step built on the device from a trace chunk
        (neo_gpu_shard_fold_step_trace): z_cpu the CPU witness (at most the bus
        base words), shout[i] = (has_lookup, key, val) and twist[i] = (has_read,
        ra, rv, has_write, wa, wv) per step; returns the step-proof words."""
        z = _u64(z_cpu)
        keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data_as(ctypes.c_void_p)

        steps = 0
        sh_ev = (_ShoutEvents * max(1, len(shout)))()
        for i, (has, key, val) in enumerate(shout):
            steps = len(has)
            sh_ev[i] = _ShoutEvents(arr(has, np.uint8), arr(key, np.uint64), arr(val, np.uint64))
        tw_ev = (_TwistEvents * max(1, len(twist)))()
        for i, (hr, ra, rv, hw, wa, wv) in enumerate(twist):
            steps = len(hr)
            tw_ev[i] = _TwistEvents(arr(hr, np.uint8), arr(ra, np.uint64), arr(rv, np.uint64), arr(hw, np.uint8),
                                    arr(wa, np.uint64), arr(wv, np.uint64))
        chunk = _TraceChunk(steps, ctypes.cast(sh_ev, ctypes.c_void_p), ctypes.cast(tw_ev, ctypes.c_void_p))
        n = ctypes.c_uint64()
        if self._cap == 0:
            self._cap = 1 << 20
        out = np.empty(self._cap, np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_fold_step_trace(self.h, _p(z) if z.size else None, z.size,
                                                                  ctypes.byref(chunk), _p(out), self._cap,
                                                                  ctypes.byref(n)))
        return out[: n.value].copy()

    def fold_step_device(self, d_z_ptr: int) -> int:
        n = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.neo_gpu_shard_fold_step_device(self.h, ctypes.c_void_p(d_z_ptr), ctypes.byref(n)))
        return n.value

    STAT_NAMES = ("total", "witness", "bind", "ccs_build", "time_rounds", "ajtai_rounds", "me_outputs",
                  "rlc_dec", "val_lane", "transcript_perms", "memory_sidecar", "unused")

    def step_stats(self) -> dict:
        out = np.zeros(12, np.float64)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_step_stats(self.h, _p(out), 12))
        return {k: float(v) for k, v in zip(self.STAT_NAMES, out)}

    def set_twist_init(self, mem_idx: int, init):
        """MemInit of Twist instance mem_idx for the following steps: [(addr, value)]
        with strictly increasing addresses (empty: MemInit::Zero)."""
        a = np.array([int(x) for x, _ in init], np.uint64)
        v = np.array([int(y) % 0xFFFFFFFF00000001 for _, y in init], np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_set_twist_init(self.h, mem_idx, len(init),
                                                                 _p(a) if len(init) else None,
                                                                 _p(v) if len(init) else None))

    def val_obligations(self) -> int:
        c = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.neo_gpu_shard_val_obligations(self.h, ctypes.byref(c)))
        return int(c.value)

    def step_proof(self) -> np.ndarray:
        """The last fold step's proof in StepProof field order (neo_gpu_shard_step_proof)."""
        n = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.neo_gpu_shard_step_proof(self.h, None, 0, ctypes.byref(n)))
        out = np.empty(n.value, np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_step_proof(self.h, _p(out), n.value, ctypes.byref(n)))
        return out

    def transcript_state(self) -> np.ndarray:
        st = np.empty(8, np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_transcript_state(self.h, _p(st)))
        return st

    def checkpoint(self) -> np.ndarray:
        """The state carried to the next fold step, as bytes (neo_gpu_shard_checkpoint)."""
        n = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.neo_gpu_shard_checkpoint(self.h, None, 0, ctypes.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_checkpoint(self.h, _p(buf), buf.size, ctypes.byref(n)))
        return buf

    def restore(self, buf: np.ndarray):
        """Continue from a checkpoint of a shard with the same CCS, m_in, k_rho and memory."""
        buf = np.ascontiguousarray(buf, np.uint8)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_restore(self.h, _p(buf), buf.size))

    def ccs_digest(self) -> np.ndarray:
        d = np.empty(4, np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_shard_ccs_digest(self.h, _p(d)))
        return d

    def close(self):
        if getattr(self, "h", None):
            if self.ctx.h is not None:
                self.ctx.lib.neo_gpu_shard_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class HostTranscript:
    """The library's host transcript (neo_transcript_*), usable without a GPU."""

    def __init__(self, app_label: bytes):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.neo_transcript_new(app_label, ctypes.byref(h))
        if rc:
            raise NeoGpuError(rc, "transcript")
        self.h = h

    def append_message(self, label: bytes, msg: bytes = b""):
        buf = ctypes.create_string_buffer(msg, len(msg)) if msg else None
        self.lib.neo_transcript_append_message(self.h, label, buf, len(msg))

    def append_fields(self, label: bytes, fs):
        fs = _u64(np.asarray(fs, dtype=np.uint64).reshape(-1))
        self.lib.neo_transcript_append_fields(self.h, label, _p(fs) if fs.size else None, fs.size)

    def append_u64s(self, label: bytes, us):
        us = _u64(us)
        self.lib.neo_transcript_append_u64s(self.h, label, _p(us), us.size)

    def challenge_field(self, label: bytes) -> int:
        out = ctypes.c_uint64()
        self.lib.neo_transcript_challenge_field(self.h, label, ctypes.byref(out))
        return out.value

    def challenge_fields(self, label: bytes, n: int):
        out = np.empty(n, np.uint64)
        self.lib.neo_transcript_challenge_fields(self.h, label, n, _p(out))
        return out

    def digest32(self) -> bytes:
        out = np.empty(32, np.uint8)
        self.lib.neo_transcript_digest32(self.h, _p(out))
        return out.tobytes()

    def state(self):
        st = np.empty(8, np.uint64)
        self.lib.neo_transcript_state(self.h, _p(st))
        return st

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.neo_transcript_destroy(self.h)
            self.h = None


def ccs_digest(ccs) -> np.ndarray:
    d = np.empty(4, np.uint64)
    desc = ccs.desc()
    rc = load().neo_ccs_digest(ctypes.byref(desc), _p(d))
    if rc:
        raise NeoGpuError(rc, "ccs digest")
    return d


class Batch:
    """Many shard-prove requests on one GPU (neo_gpu_batch): n_workers host
    threads, one CUDA stream each; requests leave one FIFO queue when their
    device footprint fits the HBM budget and are proven to completion."""

    def __init__(self, device: int = 0, n_workers: int = 8, reserve_bytes: int = None):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.neo_gpu_batch_create(device, n_workers, ctypes.byref(h))
        if rc:
            raise NeoGpuError(rc, "batch creation failed")
        self.h = h
        if reserve_bytes is not None:
            self.lib.neo_gpu_batch_set_reserve(self.h, reserve_bytes)
        self._descs = []

    def submit(self, ccs, z, n_steps: int, m_in: int = 1, k_rho: int = 12,
               app_label: bytes = b"neo/shard", mem: dict = None, inits=None) -> int:
        """z: one witness for every step, or a list of n_steps witnesses (consecutive
        trace chunks) with inits[s][i] = the MemInit [(addr, value)] of Twist i
        before step s (neo_gpu_batch_submit_chunks)."""
        desc = ccs.desc()
        jid = ctypes.c_uint64()
        if isinstance(z, (list, tuple)):
            if len(z) != n_steps:
                raise ValueError("one witness per step")
            zs = np.ascontiguousarray(np.stack([_u64(v) for v in z]))
            md = _mem_desc(mem) if mem else None
            n_twist = len(mem.get("twist", [])) if mem else 0
            arr, keep = None, []
            if inits is not None and n_twist:
                arr = (MemInit * (n_steps * n_twist))()
                for s_ in range(1, n_steps):
                    for i in range(n_twist):
                        pairs = inits[s_][i]
                        a = np.array([int(x) for x, _ in pairs], np.uint64)
                        v = np.array([int(y) % 0xFFFFFFFF00000001 for _, y in pairs], np.uint64)
                        keep += [a, v]
                        e = arr[s_ * n_twist + i]
                        e.n_init, e.addr, e.val = len(pairs), _p(a) if len(pairs) else None, _p(v) if len(pairs) else None
            rc = self.lib.neo_gpu_batch_submit_chunks(self.h, ctypes.byref(desc), ctypes.byref(md) if md else None,
                                                      _p(zs), arr, n_steps, m_in, k_rho, app_label, ctypes.byref(jid))
            if rc:
                raise NeoGpuError(rc, "batch submit")
            return jid.value
        z = _u64(z)
        if mem and (mem.get("shout") or mem.get("twist")):
            md = _mem_desc(mem)
            rc = self.lib.neo_gpu_batch_submit_mem(self.h, ctypes.byref(desc), ctypes.byref(md), _p(z), n_steps, m_in,
                                                   k_rho, app_label, ctypes.byref(jid))
        else:
            rc = self.lib.neo_gpu_batch_submit(self.h, ctypes.byref(desc), _p(z), n_steps, m_in, k_rho, app_label,
                                               ctypes.byref(jid))
        if rc:
            raise NeoGpuError(rc, "batch submit")
        return jid.value

    def cancel(self, jid: int):
        """A queued request never starts; a running one stops before its next step."""
        rc = self.lib.neo_gpu_batch_cancel(self.h, jid)
        if rc:
            raise NeoGpuError(rc, "batch cancel")

    def wait_all(self, timeout_s: float = 3600.0):
        rc = self.lib.neo_gpu_batch_wait_all(self.h, timeout_s * 1e3)
        if rc:
            raise NeoGpuError(rc, "batch wait timed out")

    def job_info(self, jid: int) -> dict:
        t = np.zeros(3, np.float64)
        st = np.zeros(8, np.uint64)
        status = ctypes.c_int()
        self.lib.neo_gpu_batch_job_info(self.h, jid, _p(t), _p(st), ctypes.byref(status))
        info = {"latency_ms": float(t[0]), "queue_ms": float(t[1]), "submit_ms": float(t[2]),
                "transcript_state": st, "status": status.value}
        if status.value < 0:
            buf = ctypes.create_string_buffer(512)
            self.lib.neo_gpu_batch_job_error(self.h, jid, buf, 512)
            info["error"] = buf.value.decode(errors="replace")
        return info

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.neo_gpu_batch_kernel_launches(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.neo_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
