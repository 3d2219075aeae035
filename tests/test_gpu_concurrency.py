"""Host threads that drive the library concurrently, each with its own context
(the batch engine's worker model)."""
import threading

import numpy as np
import pytest

from tests.helpers import ccs_case, ELL_D, D_SC, XS

pytestmark = pytest.mark.gpu


def _ajtai_phase_oracle(ctx, ell, k, seed):
    """A Pi_CCS oracle with k instances whose row rounds are done (the next
    evaluations run the Ajtai-phase kernel), and its round polynomial there."""
    from nightstream_b200.gpu import GpuCcsOracle
    ccs, z, Z, ch, chals = ccs_case(ell, k, True, seed=seed)
    g = GpuCcsOracle(ctx, ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D,
                     ell, D_SC)
    for r in range(ell):
        g.evals_at(XS)
        g.fold(chals[r])
    return g, g.evals_at(XS)


def test_concurrent_kernels_with_different_shared_memory():
    """The Ajtai-phase kernel takes k (1 + t) 54 K values of dynamic shared
    memory: 4.3 KB at k = 1 (a shard's first step), 56 KB at k = 13 (a steady
    step).  Its shared-memory limit is one process-wide attribute of the
    function, so two threads evaluating k = 1 and k = 13 oracles in tight loops
    must never see a launch fail, and every evaluation repeats the first."""
    from nightstream_b200.gpu import Context
    ell, iters = 10, 1500
    ctxs = [Context(0), Context(0)]
    cases = [_ajtai_phase_oracle(ctxs[0], ell, 1, 31), _ajtai_phase_oracle(ctxs[1], ell, 13, 32)]
    errors = []
    start = threading.Barrier(len(cases))

    def hammer(g, expect):
        try:
            start.wait()
            for i in range(iters):
                ys = g.evals_at(XS)
                if not np.array_equal(ys, expect):
                    errors.append(f"k={g.k}: evaluation {i} differs")
                    return
        except Exception as e:  # a failed launch raises NeoGpuError
            errors.append(f"k={g.k}: {e!r}")

    threads = [threading.Thread(target=hammer, args=c) for c in cases]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for g, _ in cases:
        g.close()
    for c in ctxs:
        c.close()
    assert not errors, errors
