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


def test_verifier_accepts_gpu_memory_chunks(ctx):
    """Three consecutive chunks of one trace proven by the CUDA library (one
    Shout table of 2^10 entries, one Twist memory of 2^8 cells, 64 trace steps
    per fold step) pass every memory-sidecar check of the verifier."""
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(13, 21, 3, 64, 10, 8)
    ctx.pp_generate(bytes(range(1, 33)), 16, 1 << 13, 1)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/gpu-verify-mem", mem=mem)
    v = OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/gpu-verify-mem", mem=mem)
    for c in range(3):
        if c:
            g.set_twist_init(0, inits[c][0])
            v.set_twist_init(0, inits[c][0])
        assert v.verify_step(zs[c][:1], g.fold_step(zs[c]))
    assert len(v.val_obligations) == g.val_obligations() == 36
    g.close()


def test_verifier_accepts_full_size_memory_chunks(ctx):
    """The single-shard-with-memory workload at its full size: n = m = 2^16,
    1024 trace steps per fold step, a Twist memory of 2^12 cells and a Shout
    table of 2^16 entries; three consecutive chunks proven by the CUDA library
    pass every check of the verifier restatement."""
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(16, 1234, 3, 1024, 16, 12)
    ctx.pp_generate(bytes(range(7, 39)), 16, 1 << 16, 1)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/full-verify", mem=mem)
    v = OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/full-verify", mem=mem)
    for c in range(3):
        if c:
            g.set_twist_init(0, inits[c][0])
            v.set_twist_init(0, inits[c][0])
        assert v.verify_step(zs[c][:1], g.fold_step(zs[c]))
    g.close()


def test_verifier_accepts_large_shard_chunks(ctx):
    """The large single shard: n = m = 2^20, 2^14 trace steps per fold step
    (a 2^18-step trace folds in 16 steps), a Twist memory of 2^16 cells and a
    Shout table of 2^20 entries (59 bus columns). Two consecutive chunks
    proven by the CUDA library pass every check of the verifier restatement."""
    import time
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(20, 4321, 2, 1 << 14, 20, 16)
    ctx.pp_generate(bytes(range(3, 35)), 16, 1 << 20, 1)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/large-verify", mem=mem)
    v = OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/large-verify", mem=mem)
    for c in range(2):
        if c:
            g.set_twist_init(0, inits[c][0])
            v.set_twist_init(0, inits[c][0])
        t0 = time.perf_counter()
        P = g.fold_step(zs[c])
        t1 = time.perf_counter()
        assert v.verify_step(zs[c][:1], P)
        print(f"large shard chunk {c}: GPU fold step {1e3 * (t1 - t0):.0f} ms, verify {time.perf_counter() - t1:.1f} s")
    g.close()


@pytest.mark.parametrize("memory", [False, True])
def test_step_proof_struct_order_matches_verifier(ctx, memory):
    """neo_gpu_shard_step_proof (StepProof in struct order) equals, word for
    word, the struct the verifier restatement derives from the transcript-order
    proof, and verify_step_struct accepts it, step after step."""
    from oracle.step_proof import write_step
    if memory:
        ccs, zs, mem, inits = synth.make_memory_workload_chunks(11, 6, 3, 32, 8, 6)
    else:
        ccs, z = synth.make_r1cs(10, 9)
        zs, mem, inits = [z] * 3, None, None
    ctx.pp_generate(bytes(range(9, 41)), 16, ccs.m, 1)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/struct-gpu", mem=mem)
    v1 = OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/struct-gpu", mem=mem)
    v2 = OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/struct-gpu", mem=mem)
    for c in range(3):
        if c and inits:
            for s_ in (g, v1, v2):
                s_.set_twist_init(0, inits[c][0])
        P = g.fold_step(zs[c])
        S = g.step_proof()
        rec = {}
        assert v1.verify_step(zs[c][:1], P, record=rec)
        assert np.array_equal(S, write_step(rec, 16, 64)), f"step {c}: first mismatch at word {int(np.argmax(S != write_step(rec, 16, 64)))}"
        assert v2.verify_step_struct(zs[c][:1], S)
    g.close()
