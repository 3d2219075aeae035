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


def test_batch_trace_chunks_equal_oracle(ctx):
    """Memory shards whose fold steps prove consecutive chunks of one trace
    (neo_gpu_batch_submit_chunks: per-step witness and Twist MemInit), mixed
    with a main-lane shard, end in the oracle's transcript state."""
    cfg = [(10, 16), (12, 32), (11, 16)]
    steps = 3
    shards = [synth.make_memory_workload_chunks(ell, 700 + i, steps, chunk, 8, 6) for i, (ell, chunk) in enumerate(cfg)]
    ccs_m, z_m = synth.make_r1cs(11, 777)
    for ell in sorted({c[0] for c in cfg} | {11}):
        pp = np.random.default_rng(3000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        ctx.pp_upload(pp)
    expect = []
    for i, (ccs, zs, mem, inits) in enumerate(shards):
        ell = cfg[i][0]
        pp = np.random.default_rng(3000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
        o = OracleShard(ccs, pp, app_label=b"neo/cbatch-%d" % i, mem=mem)
        for c in range(steps):
            if c:
                o.set_twist_init(0, inits[c][0])
            o.fold_step(zs[c])
        expect.append(o.tr.state())
    pp = np.random.default_rng(3011).integers(0, Q, size=(16, 1 << 11, 54), dtype=np.uint64)
    o = OracleShard(ccs_m, np.random.default_rng(3000 + 11).integers(0, Q, size=(16, 1 << 11, 54), dtype=np.uint64),
                    app_label=b"neo/cbatch-main")
    for _ in range(steps):
        o.fold_step(z_m)
    expect_main = o.tr.state()
    mix = gpu.Batch(0, n_workers=2)
    ids = [mix.submit(ccs, zs, steps, app_label=b"neo/cbatch-%d" % i, mem=mem, inits=inits)
           for i, (ccs, zs, mem, inits) in enumerate(shards)]
    jm = mix.submit(ccs_m, [z_m] * steps, steps, app_label=b"neo/cbatch-main")
    mix.wait_all(600)
    for i, jid in enumerate(ids):
        info = mix.job_info(jid)
        assert info["status"] == 1, info
        assert np.array_equal(info["transcript_state"], expect[i]), f"chunked memory shard {i}"
    assert np.array_equal(mix.job_info(jm)["transcript_state"], expect_main)
    mix.close()


def test_batch_cancel_queued_and_running(ctx):
    """neo_gpu_batch_cancel: queued requests never start, a running one stops
    before its next fold step; all three end with NEO_ERR_CANCELLED while the
    other requests complete in their solo transcript states."""
    import time
    ell = 10
    ccs, z = synth.make_r1cs(ell, 700)
    ctx.pp_upload(np.random.default_rng(3000 + ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64))
    b = gpu.Batch(0, n_workers=1)
    long_id = b.submit(ccs, z, 200, app_label=b"neo/cancel-long")  # seconds of work, runs first
    ids = [b.submit(ccs, z, 2, app_label=b"neo/cancel-%d" % i) for i in range(4)]
    b.cancel(ids[1])
    b.cancel(ids[3])
    time.sleep(0.3)
    b.cancel(long_id)
    t0 = time.perf_counter()
    b.wait_all(600)
    assert time.perf_counter() - t0 < 60  # far less than the 200 steps would take
    info = {j: b.job_info(j) for j in [long_id] + ids}
    for j in (long_id, ids[1], ids[3]):
        assert info[j]["status"] == -6 and info[j]["error"] == "cancelled", (j, info[j]["status"])
    assert info[ids[0]]["status"] == 1 and info[ids[2]]["status"] == 1
    b.cancel(ids[0])  # finished: left as it is
    assert b.job_info(ids[0])["status"] == 1
    b.close()
    solo = gpu.Batch(0, n_workers=1)
    sids = [solo.submit(ccs, z, 2, app_label=b"neo/cancel-%d" % i) for i in (0, 2)]
    solo.wait_all(600)
    for sid, i in zip(sids, (0, 2)):
        assert np.array_equal(solo.job_info(sid)["transcript_state"], info[ids[i]]["transcript_state"])
    solo.close()
