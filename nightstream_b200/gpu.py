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
_ERRS = {1: "NEO_ERR_ARG", 2: "NEO_ERR_OOM", 3: "NEO_ERR_INVARIANT", 4: "NEO_ERR_CUDA", 5: "NEO_ERR_UNSUPPORTED"}

# symbol -> argtypes; every function returns int unless listed in _RESTYPES
SIGNATURES = {
    "neo_gpu_ctx_create": [I, P],
    "neo_gpu_ctx_destroy": [P],
    "neo_gpu_last_error": [P],
    "neo_gpu_kernel_launches": [P],
    "neo_gpu_pp_upload": [P, U32, U64, P],
    "neo_gpu_commit": [P, P, U32, U64, P],
    "neo_gpu_decomp_b2": [P, P, U64, P],
    "neo_gpu_rlc_mix": [P, P, P, U32, U64, P],
    "neo_gpu_split_b": [P, P, U64, U32, U32, P, P],
    "neo_gpu_me_y": [P, P, P, U32, U32, P, U32, P, P],
    "neo_gpu_ccs_oracle_create": [P, P, P, U32, U32, P, P, P, P, P, U32, U32, U32, P],
    "neo_gpu_ccs_oracle_evals": [P, P, U32, P],
    "neo_gpu_ccs_oracle_fold": [P, P],
    "neo_gpu_ccs_oracle_num_rounds": [P],
    "neo_gpu_ccs_oracle_degree_bound": [P],
    "neo_gpu_ccs_oracle_me_outputs": [P, P, P],
    "neo_gpu_ccs_oracle_destroy": [P],
}
_RESTYPES = {
    "neo_gpu_last_error": ctypes.c_char_p,
    "neo_gpu_kernel_launches": U64,
    "neo_gpu_ccs_oracle_num_rounds": U32,
    "neo_gpu_ccs_oracle_degree_bound": U32,
}

_lib = None


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

    def me_outputs(self):
        y = np.empty((self.k, self.t, 54, 2), np.uint64)
        ys = np.empty((self.k, self.t, 2), np.uint64)
        self.ctx.check(self.ctx.lib.neo_gpu_ccs_oracle_me_outputs(self.h, _p(y), _p(ys)))
        return y, ys

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.neo_gpu_ccs_oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
