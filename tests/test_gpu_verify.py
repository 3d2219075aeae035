"""The verifier restatement (oracle/verify.py) accepts the proofs the CUDA
library emits (neo_gpu_shard_fold_step), step after step."""
import numpy as np
import pytest

from nightstream_b200 import gpu, synth
from oracle.verify import OracleVerifier, VerifyError

Q = (1 << 64) - (1 << 32) + 1
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ell", [10, 13])
def test_verifier_accepts_gpu_proofs(ctx, ell):
    ccs, z = synth.make_r1cs(ell, 17)
    ctx.pp_generate(bytes(range(32)), 16, 1 << ell, 1)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/gpu-verify")
    v = OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/gpu-verify")
    for _ in range(3):
        assert v.verify_step(z[:1], g.fold_step(z))
    # a proof of the next step with one changed word is rejected
    P = g.fold_step(z).copy()
    P[len(P) // 2] = np.uint64((int(P[len(P) // 2]) + 1) % Q)
    with pytest.raises(VerifyError):
        v.verify_step(z[:1], P)
    g.close()
