"""Neo parameter set used on the hot path.

Mirrors ``NeoParams::goldilocks_127`` (crates/neo-params/src/lib.rs:146-166):
q = 2^64 - 2^32 + 1, eta = 81, d = 54, kappa = 16, b = 2, k_rho = 12,
B = b^k_rho = 4096, T = 216.  ``ell_d = 6`` (2^6 >= 54) and the sum-check
degree bound ``d_sc = max(deg(f) + 1, 2b + 2) = 6`` follow
crates/neo-reductions/src/engines/utils.rs:29-64.
"""
from dataclasses import dataclass

Q = (1 << 64) - (1 << 32) + 1
D = 54
ETA = 81


@dataclass(frozen=True)
class NeoParams:
    q: int = Q
    eta: int = ETA
    d: int = D
    kappa: int = 16
    b: int = 2
    k_rho: int = 12
    T: int = 216

    @property
    def B(self) -> int:
        return self.b ** self.k_rho

    @property
    def ell_d(self) -> int:
        return (self.d - 1).bit_length()

    def d_sc(self, f_degree: int) -> int:
        return max(f_degree + 1, 2 * self.b + 2)


GOLDILOCKS = NeoParams()
