"""The oracle's fold step with the shared-CPU-bus memory sidecar (one Shout
and one Twist instance) runs its sum-checks to completion on an honest trace:
every round of the CCS, Shout address, Twist address, Route-A time (seven
claims) and Twist val-eval (two, then three with rollover) sum-checks keeps
p(0) + p(1) equal to the running claim, and both DEC lanes pass their public
checks."""
import numpy as np
import pytest

from nightstream_b200 import synth
from oracle.fold import OracleShard, BusLayout

Q = (1 << 64) - (1 << 32) + 1


def test_memory_fold_steps_complete():
    ell = 10
    ccs, z, mem = synth.make_memory_workload(ell, 3, 16, 6, 5)
    assert synth.check_r1cs(ccs, z)
    pp = np.random.default_rng(ell).integers(0, Q, size=(16, 1 << ell, 54), dtype=np.uint64)
    o = OracleShard(ccs, pp, m_in=1, k_rho=12, app_label=b"neo/test-mem", mem=mem)
    sizes = [len(o.fold_step(z)) for _ in range(3)]
    assert sizes[1] == sizes[2] > sizes[0]
    assert len(o.val_obligations) == 36
    # children carry the bus openings: t + bus_cols rows of y
    assert o.acc[0]["y"].shape[0] == ccs.t + o.bus.bus_cols


def test_bus_layout_matches_reference_order():
    b = BusLayout(1024, 1, 16, [6], [5])
    assert b.shout[0]["addr_bits"] == list(range(6)) and b.shout[0]["has_lookup"] == 6 and b.shout[0]["val"] == 7
    tw = b.twist[0]
    assert tw["ra_bits"] == list(range(8, 13)) and tw["wa_bits"] == list(range(13, 18))
    assert (tw["has_read"], tw["has_write"], tw["wv"], tw["rv"], tw["inc"]) == (18, 19, 20, 21, 22)
    assert b.bus_cols == 23 and b.bus_base == 1024 - 23 * 16 and b.cell(2, 3) == b.bus_base + 35


def test_oracle_multi_chunk_trace_with_rollover_init():
    """Consecutive chunks of one trace: each fold step starts from the memory
    state the previous chunk left (MemInit per step, mem_init.rs:65-90); with a
    stale init the Twist address-lane claim (0) fails at the first round."""
    from nightstream_b200 import synth
    from oracle.fold import OracleShard
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(12, 7, 3, 32, 8, 6)
    Q = (1 << 64) - (1 << 32) + 1
    pp = np.random.default_rng(3).integers(0, Q, size=(16, 1 << 12, 54), dtype=np.uint64)
    o = OracleShard(ccs, pp, mem=mem, app_label=b"neo/chunks")
    for c in range(3):
        if c:
            o.set_twist_init(0, inits[c][0])
        o.fold_step(zs[c])
    stale = OracleShard(ccs, pp, mem=mem, app_label=b"neo/chunks")
    stale.fold_step(zs[0])
    with pytest.raises(AssertionError):
        stale.fold_step(zs[1])
    with pytest.raises(ValueError):
        stale.set_twist_init(0, [(5, 1), (5, 2)])
