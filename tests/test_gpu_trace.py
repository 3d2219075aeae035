"""Fold steps built from trace chunks on the device (neo_gpu_shard_fold_step_trace)
against the same steps proven from host-built witnesses and host MemInits
(neo_gpu_shard_fold_step + neo_gpu_shard_set_twist_init, the path the oracle
parity tests cover): every proof word and the transcript state equal, over
consecutive chunks whose Twist writes revisit addresses inside a chunk, a
partial last chunk, and the reference's build errors."""
import numpy as np
import pytest

from nightstream_b200 import gpu, synth

pytestmark = pytest.mark.gpu

Q = (1 << 64) - (1 << 32) + 1
ELL, STEPS, SE, TE = 12, 64, 8, 6  # R1CS 2^12, 64 trace steps per fold step, Shout 2^8, Twist 2^6


def _bits(rows):
    return sum(rows[b].astype(np.uint64) << np.uint64(b) for b in range(rows.shape[0]))


def _events(z, m, steps):
    """The trace events a chunk's bus tail encodes (column order of the shared
    CPU bus: Shout [addr bits, has_lookup, val], Twist [ra bits, wa bits,
    has_read, has_write, wv, rv, inc])."""
    cols = (SE + 2) + (2 * TE + 5)
    base = m - cols * steps
    bus = z[base:].reshape(cols, steps)
    s = bus[:SE + 2]
    t = bus[SE + 2:]
    shout = [(s[SE].astype(np.uint8), _bits(s[:SE]), s[SE + 1])]
    twist = [(t[2 * TE].astype(np.uint8), _bits(t[:TE]), t[2 * TE + 3], t[2 * TE + 1].astype(np.uint8),
              _bits(t[TE:2 * TE]), t[2 * TE + 2])]
    return base, shout, twist


@pytest.fixture(scope="module")
def workload():
    return synth.make_memory_workload_chunks(ELL, 41, 4, STEPS, SE, TE)


def _pair(ctx, ccs, mem):
    a = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/trace", mem=mem)
    b = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/trace", mem=mem)
    return a, b


def test_trace_steps_equal_witness_steps(ctx, workload):
    ccs, zs, mem, inits = workload
    m = 1 << ELL
    ctx.pp_upload(np.random.default_rng(3).integers(0, Q, size=(16, m, 54), dtype=np.uint64))
    a, b = _pair(ctx, ccs, mem)
    for c in range(len(zs)):
        if c:
            a.set_twist_init(0, inits[c][0])
        pa = a.fold_step(zs[c])
        base, shout, twist = _events(zs[c], m, STEPS)
        # writes revisit addresses inside the chunk (the increment sort's case)
        wa = twist[0][4][twist[0][3] == 1]
        assert len(np.unique(wa)) < len(wa)
        pb = b.fold_step_trace(zs[c][:base], shout, twist)
        assert np.array_equal(pa, pb), f"chunk {c}: first difference at word {int(np.argmax(pa != pb))}"
        assert np.array_equal(a.transcript_state(), b.transcript_state())
    a.close()
    b.close()


def test_partial_last_chunk_and_rebuilt_memory(ctx, workload):
    """A last chunk with fewer steps than the shard's equals the witness whose
    unused bus cells are zero; a MemInit set between trace steps replaces the
    device memory."""
    ccs, zs, mem, inits = workload
    m = 1 << ELL
    ctx.pp_upload(np.random.default_rng(3).integers(0, Q, size=(16, m, 54), dtype=np.uint64))
    a, b = _pair(ctx, ccs, mem)
    for c in range(2):
        if c:
            a.set_twist_init(0, inits[c][0])
        base, shout, twist = _events(zs[c], m, STEPS)
        assert np.array_equal(a.fold_step(zs[c]), b.fold_step_trace(zs[c][:base], shout, twist))
    # chunk 2 truncated to 50 steps
    keep = 50
    z = zs[2].copy()
    cols = (SE + 2) + (2 * TE + 5)
    bus = z[m - cols * STEPS:].reshape(cols, STEPS)
    bus[:, keep:] = 0
    a.set_twist_init(0, inits[2][0])
    base, shout, twist = _events(z, m, STEPS)
    shout = [tuple(x[:keep] for x in ev) for ev in shout]
    twist = [tuple(x[:keep] for x in ev) for ev in twist]
    assert np.array_equal(a.fold_step(z), b.fold_step_trace(z[:base], shout, twist))
    # an explicit MemInit between trace steps: both shards start chunk 3 from
    # it (reads and increments of the chunk replayed against that memory)
    init = [(1, 5), (7, 11)]
    a.set_twist_init(0, init)
    b.set_twist_init(0, init)
    z3 = zs[3].copy()
    bus3 = z3[m - cols * STEPS:].reshape(cols, STEPS)
    t = bus3[SE + 2:]
    hr, ra, hw, wa, wv = t[2 * TE], _bits(t[:TE]), t[2 * TE + 1], _bits(t[TE:2 * TE]), t[2 * TE + 2]
    memory = dict(init)
    for j in range(STEPS):
        t[2 * TE + 3, j] = memory.get(int(ra[j]), 0) if hr[j] else 0
        if hw[j]:
            t[2 * TE + 4, j] = (int(wv[j]) - memory.get(int(wa[j]), 0)) % Q
            memory[int(wa[j])] = int(wv[j])
        else:
            t[2 * TE + 4, j] = 0
    base, shout, twist = _events(z3, m, STEPS)
    assert np.array_equal(a.fold_step(z3), b.fold_step_trace(z3[:base], shout, twist))
    assert np.array_equal(a.transcript_state(), b.transcript_state())
    a.close()
    b.close()


def test_trace_step_errors(ctx, workload):
    ccs, zs, mem, inits = workload
    m = 1 << ELL
    ctx.pp_upload(np.random.default_rng(3).integers(0, Q, size=(16, m, 54), dtype=np.uint64))
    sh = gpu.Shard(ctx, ccs, m_in=1, k_rho=12, app_label=b"neo/trace", mem=mem)
    base, shout, twist = _events(zs[0], m, STEPS)
    bad_flag = [tuple(x.copy() for x in twist[0])]
    bad_flag[0][0][3] = 2
    bad_addr = [tuple(x.copy() for x in twist[0])]
    bad_addr[0][3][:] = 1
    bad_addr[0][4][5] = 1 << TE
    too_long = [tuple(np.concatenate([x, x[:1]]) for x in shout[0])]
    for args in ((zs[0][:base], shout, bad_flag), (zs[0][:base], shout, bad_addr),
                 (zs[0][:base + 1], shout, twist), (zs[0][:base], too_long, [tuple(np.concatenate([x, x[:1]])
                                                                                  for x in twist[0])])):
        with pytest.raises(gpu.NeoGpuError) as e:
            sh.fold_step_trace(*args)
        assert e.value.code == 1
    # the shard is still usable
    assert len(sh.fold_step_trace(zs[0][:base], shout, twist)) > 0
    sh.close()
