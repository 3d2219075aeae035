"""Whole fold steps through the C ABI (neo_gpu_shard_fold_step) against the
oracle's fold-step restatement: every proof word and the transcript state must
be identical, for the first step (k = 1) and steady-state steps (k = 13)."""
import numpy as np
import pytest

from oracle.fold import OracleShard
from nightstream_b200 import gpu, synth

Q = (1 << 64) - (1 << 32) + 1
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ell,steps", [(6, 3), (10, 3)])
def test_fold_steps_match_oracle(ctx, ell, steps):
    ccs, z = synth.make_r1cs(ell, 21)
    pp = np.random.default_rng(ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/test-shard")
    o = OracleShard(ccs, pp, m_in=1, k_rho=12, app_label=b"neo/test-shard")
    assert np.array_equal(g.ccs_digest(), o.digest)
    for s in range(steps):
        pg = g.fold_step(z)
        po = o.fold_step(z)
        assert pg.shape == po.shape, f"step {s}: proof length"
        assert np.array_equal(pg, po), f"step {s}: first mismatch at word {int(np.argmax(pg != po))}"
        assert np.array_equal(g.transcript_state(), o.tr.state()), f"step {s}: transcript state"
    g.close()


def test_fold_step_rejects_unsatisfied_witness(ctx):
    ccs, z = synth.make_r1cs(6, 22)
    pp = np.random.default_rng(1).integers(0, Q, size=(16, 64, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    g = gpu.Shard(ctx, ccs)
    bad = z.copy()
    bad[3] = (int(bad[3]) + 1) % Q
    with pytest.raises(gpu.NeoGpuError) as e:
        g.fold_step(bad)
    assert e.value.code == 3  # NEO_ERR_INVARIANT: sum-check p(0)+p(1) check
    g.close()


@pytest.mark.parametrize("ell,steps,chunk,shout_ell,twist_ell", [(10, 3, 16, 6, 5), (12, 2, 64, 8, 6)])
def test_memory_fold_steps_match_oracle(ctx, ell, steps, chunk, shout_ell, twist_ell):
    """Fold steps with the shared-CPU-bus memory sidecar (one Shout table, one
    Twist memory): every proof word (address pre-time rounds, the seven Route-A
    time claims, bus openings, val-eval batch, both RLC/DEC lanes) and the
    transcript state match the oracle, for the first step and with rollover."""
    ccs, z, mem = synth.make_memory_workload(ell, 5, chunk, shout_ell, twist_ell)
    pp = np.random.default_rng(ell + 1).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/test-mem", mem=mem)
    o = OracleShard(ccs, pp, m_in=1, k_rho=12, app_label=b"neo/test-mem", mem=mem)
    for s in range(steps):
        pg = g.fold_step(z)
        po = o.fold_step(z)
        assert pg.shape == po.shape, f"step {s}: proof length {pg.shape} vs {po.shape}"
        assert np.array_equal(pg, po), f"step {s}: first mismatch at word {int(np.argmax(pg != po))}"
        assert np.array_equal(g.transcript_state(), o.tr.state()), f"step {s}: transcript state"
    assert g.val_obligations() == 12 * steps
    g.close()


@pytest.mark.parametrize("ell,chunks,chunk,shout_ell,twist_ell", [(12, 3, 32, 8, 6), (13, 3, 64, 10, 8)])
def test_memory_multi_chunk_trace_matches_oracle(ctx, ell, chunks, chunk, shout_ell, twist_ell):
    """Consecutive chunks of one trace, each step starting from the memory state
    the previous chunk left (neo_gpu_shard_set_twist_init): every proof word and
    the transcript state match the oracle; a stale init is rejected (the Twist
    address-lane claim 0 fails at its first round, NEO_ERR_INVARIANT)."""
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(ell, 9, chunks, chunk, shout_ell, twist_ell)
    pp = np.random.default_rng(ell + 3).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    g = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/test-chunks", mem=mem)
    o = OracleShard(ccs, pp, m_in=1, k_rho=12, app_label=b"neo/test-chunks", mem=mem)
    for c in range(chunks):
        if c:
            g.set_twist_init(0, inits[c][0])
            o.set_twist_init(0, inits[c][0])
        pg, po = g.fold_step(zs[c]), o.fold_step(zs[c])
        assert np.array_equal(pg, po), f"chunk {c}: first mismatch at word {int(np.argmax(pg != po))}"
        assert np.array_equal(g.transcript_state(), o.tr.state()), f"chunk {c}: transcript state"
    g.close()
    stale = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/test-chunks", mem=mem)
    stale.fold_step(zs[0])
    with pytest.raises(gpu.NeoGpuError) as e:
        stale.fold_step(zs[1])
    assert e.value.code == 3
    with pytest.raises(gpu.NeoGpuError):
        stale.set_twist_init(0, [(7, 1), (3, 2)])
    with pytest.raises(gpu.NeoGpuError):
        stale.set_twist_init(1, [])
    stale.close()


def test_memory_fold_rejects_bad_read(ctx):
    """A read value that disagrees with memory breaks the Twist checks: the
    prover stops with the invariant status instead of emitting a proof."""
    ccs, z, mem = synth.make_memory_workload(10, 6, 16, 6, 5)
    pp = np.random.default_rng(3).integers(0, Q, size=(16, 1 << 10, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    g = gpu.Shard(ctx, ccs, mem=mem)
    bus_cols = (6 + 2) + (2 * 5 + 5)
    base = (1 << 10) - bus_cols * 16
    rv_col = 8 + 2 * 5 + 3
    bad = z.copy()
    bad[base + rv_col * 16 + 3] = (int(bad[base + rv_col * 16 + 3]) + 1) % Q
    with pytest.raises(gpu.NeoGpuError) as e:
        g.fold_step(bad)
    assert e.value.code == 3
    g.close()


@pytest.mark.parametrize("case", [
    dict(shout_ell=[6], twist_ell=[5, 4], init_cells=0),           # two Twist memories, MemInit::Zero
    dict(shout_ell=[6, 6], twist_ell=[5], lookup_rate=0.0),        # no lookups: sampled r_addr, no sum-check
    dict(shout_ell=[6, 6], twist_ell=[], lookup_rate=0.5),         # Shout only, half the steps look up
    dict(shout_ell=[], twist_ell=[5], rw_rate=0.6),                # Twist only, sparse reads / writes
])
def test_memory_fold_instance_mixes(ctx, case):
    ell = 10
    ccs, z, mem = synth.make_memory_workload(ell, 9, 8, **case)
    pp = np.random.default_rng(ell + 7).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    g = gpu.Shard(ctx, ccs, mem=mem, app_label=b"neo/test-mix")
    o = OracleShard(ccs, pp, mem=mem, app_label=b"neo/test-mix")
    for s in range(2):
        pg, po = g.fold_step(z), o.fold_step(z)
        assert pg.shape == po.shape and np.array_equal(pg, po), f"step {s}"
        assert np.array_equal(g.transcript_state(), o.tr.state())
    g.close()
