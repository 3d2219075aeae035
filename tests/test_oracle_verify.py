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


@pytest.fixture(scope="module")
def mem_proofs():
    """Three consecutive chunks of one trace (one Shout table, one Twist memory)."""
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(12, 7, 3, 32, 8, 6)
    pp = np.random.default_rng(3).integers(0, Q, size=(16, 1 << 12, 54), dtype=np.uint64)
    sh = OracleShard(ccs, pp, mem=mem, app_label=b"neo/verify-mem")
    Ps = []
    for c in range(3):
        if c:
            sh.set_twist_init(0, inits[c][0])
        Ps.append(sh.fold_step(zs[c]))
    return ccs, zs, mem, inits, Ps


def _mem_verifier(ccs, mem):
    return OracleVerifier(ccs, mem=mem, app_label=b"neo/verify-mem")


def _verify_chunks(v, zs, inits, Ps, upto):
    for c in range(upto):
        if c:
            v.set_twist_init(0, inits[c][0])
        v.verify_step(zs[c][:1], Ps[c])


def test_verifier_accepts_memory_chunks(mem_proofs):
    """Shout / Twist address pre-time, the seven Route-A time claims with their
    terminal values at the bus openings, the Twist val-eval batch with rollover
    (Init_i(r_addr) = Init_{i-1}(r_addr) + PrevTotal), both lanes."""
    ccs, zs, mem, inits, Ps = mem_proofs
    v = _mem_verifier(ccs, mem)
    _verify_chunks(v, zs, inits, Ps, 3)
    assert len(v.val_obligations) == 36


def test_verifier_rejects_a_stale_memory_init(mem_proofs):
    ccs, zs, mem, inits, Ps = mem_proofs
    v = _mem_verifier(ccs, mem)
    v.verify_step(zs[0][:1], Ps[0])
    with pytest.raises(VerifyError):  # the verifier still holds chunk 0's MemInit
        v.verify_step(zs[1][:1], Ps[1])


@pytest.mark.parametrize("frac", [0.0005, 0.002, 0.01, 0.03, 0.1, 0.3, 0.5, 0.8, 0.99])
def test_verifier_rejects_a_changed_memory_step_word(mem_proofs, frac):
    ccs, zs, mem, inits, Ps = mem_proofs
    v = _mem_verifier(ccs, mem)
    _verify_chunks(v, zs, inits, Ps, 2)
    v.set_twist_init(0, inits[2][0])
    bad = np.array(Ps[2], np.uint64).copy()
    pos = 864 + int(frac * (len(bad) - 864))
    bad[pos] = np.uint64((int(bad[pos]) + 1) % Q)
    with pytest.raises(VerifyError):
        v.verify_step(zs[2][:1], bad)
