"""Seeded test cases shared by the CPU and GPU test modules."""
import numpy as np

import oracle as O
from nightstream_b200 import synth

ELL_D = 6
D_SC = 6
XS = np.array([[i, 0] for i in range(D_SC + 1)], np.uint64)


def ccs_case(ell, k, with_inputs, seed=7):
    """R1CS of 2^ell rows, MCS witness digits + (k-1) random digit matrices."""
    ccs, z = synth.make_r1cs(ell, seed)
    rng = np.random.default_rng(seed + 100)
    Z0 = O.decomp_b2(z)
    Zs = [Z0] + [rng.integers(-1, 2, size=(54, 1 << ell)).astype(np.int8) for _ in range(k - 1)]
    Z = np.stack(Zs)
    ch = dict(
        alpha=synth.uniform_k(rng, ELL_D), beta_a=synth.uniform_k(rng, ELL_D),
        beta_r=synth.uniform_k(rng, ell), gamma=synth.uniform_k(rng, 1)[0],
        r_inputs=synth.uniform_k(rng, ell) if with_inputs else None,
    )
    chals = synth.uniform_k(rng, ell + ELL_D)
    return ccs, z, Z, ch, chals


def kadd(a, b):
    q = (1 << 64) - (1 << 32) + 1
    return np.array([(int(a[0]) + int(b[0])) % q, (int(a[1]) + int(b[1])) % q], np.uint64)
