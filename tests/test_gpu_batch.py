"""Batched proving: every shard's result in the mix (several workers, uneven
sizes, interleaved steps) equals the oracle's and its own solo result."""
import numpy as np
import pytest

from oracle.fold import OracleShard
from nightstream_b200 import gpu, synth

Q = (1 << 64) - (1 << 32) + 1
pytestmark = pytest.mark.gpu


def test_batch_results_equal_solo_and_oracle(ctx):
    sizes = [6, 8, 7, 6, 8]
    steps = 3
    shards = [synth.make_r1cs(ell, 500 + i) for i, ell in enumerate(sizes)]
    for ell in sorted(set(sizes)):
        pp = np.random.default_rng(1000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        ctx.pp_upload(pp)
    expect = []
    for i, (ccs, z) in enumerate(shards):
        ell = sizes[i]
        pp = np.random.default_rng(1000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        o = OracleShard(ccs, pp, app_label=b"neo/batch-%d" % i)
        for _ in range(steps):
            o.fold_step(z)
        expect.append(o.tr.state())
    mix = gpu.Batch(0, n_workers=3)
    ids = [mix.submit(ccs, z, steps, app_label=b"neo/batch-%d" % i) for i, (ccs, z) in enumerate(shards)]
    mix.wait_all(600)
    for i, jid in enumerate(ids):
        info = mix.job_info(jid)
        assert info["status"] == 1
        assert np.array_equal(info["transcript_state"], expect[i]), f"shard {i} in the mix"
    mix.close()
    solo = gpu.Batch(0, n_workers=1)
    jid = solo.submit(shards[2][0], shards[2][1], steps, app_label=b"neo/batch-2")
    solo.wait_all(600)
    assert np.array_equal(solo.job_info(jid)["transcript_state"], expect[2])
    solo.close()


def test_batch_memory_shards_equal_oracle(ctx):
    """Shards with the memory sidecar in the mix (uneven sizes, interleaved
    steps on three workers) end in the oracle's transcript state."""
    cfg = [(10, 16), (11, 16), (10, 8), (12, 32)]
    steps = 2
    shards = [synth.make_memory_workload(ell, 600 + i, chunk, 8, 6) for i, (ell, chunk) in enumerate(cfg)]
    for ell in sorted({c[0] for c in cfg}):
        pp = np.random.default_rng(2000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        ctx.pp_upload(pp)
    expect = []
    for i, (ccs, z, mem) in enumerate(shards):
        ell = cfg[i][0]
        pp = np.random.default_rng(2000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        o = OracleShard(ccs, pp, app_label=b"neo/mbatch-%d" % i, mem=mem)
        for _ in range(steps):
            o.fold_step(z)
        expect.append(o.tr.state())
    mix = gpu.Batch(0, n_workers=3)
    ids = [mix.submit(ccs, z, steps, app_label=b"neo/mbatch-%d" % i, mem=mem)
           for i, (ccs, z, mem) in enumerate(shards)]
    mix.wait_all(600)
    for i, jid in enumerate(ids):
        info = mix.job_info(jid)
        assert info["status"] == 1, info
        assert np.array_equal(info["transcript_state"], expect[i]), f"memory shard {i} in the mix"
    mix.close()
