"""Failure detection without a GPU fault: a bounded device wait that runs out
is reported as a status the host reads, and the context keeps working."""
import numpy as np
import pytest

import oracle as O
from nightstream_b200 import gpu

pytestmark = pytest.mark.gpu
Q = (1 << 64) - (1 << 32) + 1


def test_bounded_wait_times_out_and_context_survives(ctx):
    ctx.wait_probe(True)  # the flag is set: the wait ends at once
    with pytest.raises(gpu.NeoGpuError) as e:
        ctx.wait_probe(False, spin_limit=2000)  # nothing sets the flag: ~2 ms, then the error word
    assert e.value.code == 4 and "timed out" in str(e.value)
    ctx.wait_probe(True)  # the error word was read and cleared
    # the same context still computes: a commitment equals the oracle's
    m = 256
    pp = np.random.default_rng(77).integers(0, Q, size=(16, m, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    Z = np.random.default_rng(78).integers(-1, 2, size=(54, m)).astype(np.int8)
    assert np.array_equal(ctx.commit(Z), O.commit_digits(pp, Z))


def test_wait_probe_rejects_unbounded_limits(ctx):
    for bad in (0, (1 << 20) + 1):
        with pytest.raises(gpu.NeoGpuError) as e:
            ctx.wait_probe(False, spin_limit=bad)
        assert e.value.code == 1
