"""Checkpoint / resume of a shard prover (neo_gpu_shard_checkpoint /
neo_gpu_shard_restore): a shard restored from a checkpoint proves its next
fold step exactly as the shard it was taken from."""
import numpy as np
import pytest

from nightstream_b200 import gpu, synth

pytestmark = pytest.mark.gpu
Q = (1 << 64) - (1 << 32) + 1


def _pp(ctx, ell, seed):
    ctx.pp_upload(np.random.default_rng(seed).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64))


def test_memory_shard_resumes_from_every_step(ctx):
    """Consecutive trace chunks (Twist rollover, val lane, per-step MemInit):
    before each step the shard is checkpointed and restored into a new shard
    in another context under another app label; the restored shard's step
    gives the same proof words, transcript state and obligation count."""
    ell, chunks, chunk = 12, 4, 32
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(ell, 21, chunks, chunk, 8, 6)
    _pp(ctx, ell, 5)
    ctx2 = gpu.Context(0)
    a = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/ckpt", mem=mem)
    sizes = []
    for c in range(chunks):
        if c:
            a.set_twist_init(0, inits[c][0])
        ck = a.checkpoint()
        sizes.append(ck.size)
        pa = a.fold_step(zs[c])
        b = gpu.Shard(ctx2, ccs, m_in=1, k_rho=12, app_label=b"neo/another-label", mem=mem)
        b.restore(ck)
        pb = b.fold_step(zs[c])
        assert np.array_equal(pa, pb), f"chunk {c}: first mismatch at word {int(np.argmax(pa != pb))}"
        assert np.array_equal(a.transcript_state(), b.transcript_state()), f"chunk {c}"
        assert a.val_obligations() == b.val_obligations()
        b.close()
    # step 0 carries no accumulator; later checkpoints carry 12 digit planes,
    # the previous MCS witness and the previous bus columns
    assert sizes[0] < sizes[1] == sizes[2] == sizes[3]
    a.close()
    ctx2.close()


def test_main_lane_shard_resumes_and_rejects_foreign_checkpoints(ctx):
    """Without memory: resume after two steps matches; a checkpoint of another
    CCS, and a truncated one, are refused (NEO_ERR_ARG) and leave the target
    shard able to prove its own steps."""
    ell = 10
    ccs, z = synth.make_r1cs(ell, 8)
    other, _ = synth.make_r1cs(ell, 9)
    _pp(ctx, ell, 6)
    a = gpu.Shard(ctx, ccs, app_label=b"neo/ckpt-main")
    ref = gpu.Shard(ctx, ccs, app_label=b"neo/ckpt-main")
    for _ in range(2):
        a.fold_step(z)
        ref.fold_step(z)
    ck = a.checkpoint()
    b = gpu.Shard(ctx, ccs, app_label=b"neo/x")
    b.restore(ck)
    for _ in range(2):
        pa, pb = a.fold_step(z), b.fold_step(z)
        assert np.array_equal(pa, pb)
        assert np.array_equal(a.transcript_state(), b.transcript_state())
    c = gpu.Shard(ctx, other, app_label=b"neo/ckpt-main")
    with pytest.raises(gpu.NeoGpuError) as e:
        c.restore(ck)
    assert e.value.code == 1
    with pytest.raises(gpu.NeoGpuError) as e:
        ref.restore(ck[: ck.size // 2])
    assert e.value.code == 1
    # the refused restore changed nothing: ref continues its own chain, equal to a's
    p_ref = ref.fold_step(z)
    a2 = gpu.Shard(ctx, ccs, app_label=b"neo/ckpt-main")
    for _ in range(3):
        p_a2 = a2.fold_step(z)
    assert np.array_equal(p_ref, p_a2)
    for s in (a, b, c, ref, a2):
        s.close()
