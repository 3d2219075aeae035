"""The verifier restatement (oracle/verify.py, shard.rs:2482-2900 and
shard.rs:1333-1420) accepts the oracle prover's step proofs and rejects any
changed proof word."""
import numpy as np
import pytest

from nightstream_b200 import synth
from oracle.fold import OracleShard
from oracle.verify import OracleVerifier, VerifyError

Q = (1 << 64) - (1 << 32) + 1
ELL = 10


@pytest.fixture(scope="module")
def proofs():
    ccs, z = synth.make_r1cs(ELL, 5)
    pp = np.random.default_rng(3).integers(0, Q, size=(16, 1 << ELL, 54), dtype=np.uint64)
    sh = OracleShard(ccs, pp, m_in=1, k_rho=12, app_label=b"neo/verify-test")
    return ccs, z, [sh.fold_step(z) for _ in range(3)]


def _verifier(ccs):
    return OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/verify-test")


def test_verifier_accepts_prover_steps(proofs):
    ccs, z, Ps = proofs
    v = _verifier(ccs)
    for P in Ps:
        assert v.verify_step(z[:1], P)
    assert len(v.acc) == 12


# step-1 proof layout (k = 13, ell_n = 10, d_sc = 6): c_mcs [0, 864), T [864, 866),
# time rounds [866, 1006), Ajtai rounds [1006, 1090), running [1090, 1092),
# y [1092, 6708), y_scalars [6708, 6812), rhos [6812, 7514), c_parent [7514, 8378),
# 12 children x (c 864 + y 432) [8378, 23930)
@pytest.mark.parametrize("pos", [5, 864, 870, 1010, 1090, 1100, 6710, 6820, 7600, 8400, 9300, 23929])
def test_verifier_rejects_a_changed_word(proofs, pos):
    ccs, z, Ps = proofs
    assert len(Ps[1]) == 23930
    v = _verifier(ccs)
    v.verify_step(z[:1], Ps[0])
    bad = np.array(Ps[1], np.uint64).copy()
    bad[pos] = np.uint64((int(bad[pos]) + 1) % Q)
    with pytest.raises(VerifyError):
        v.verify_step(z[:1], bad)


def test_verifier_rejects_wrong_public_input(proofs):
    ccs, z, Ps = proofs
    v = _verifier(ccs)
    with pytest.raises(VerifyError):
        v.verify_step(np.array([2], np.uint64), Ps[0])


def test_verifier_rejects_truncated_and_padded_proofs(proofs):
    ccs, z, Ps = proofs
    with pytest.raises(VerifyError):
        _verifier(ccs).verify_step(z[:1], Ps[0][:-1])
    with pytest.raises(VerifyError):
        _verifier(ccs).verify_step(z[:1], np.concatenate([Ps[0], np.zeros(1, np.uint64)]))
