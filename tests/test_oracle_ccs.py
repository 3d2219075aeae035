"""Pins the C restatement of the Pi_CCS oracle against the paper-exact Q
(crates/neo-reductions/tests/optimized_oracle_row_stream_smoke.rs:44-150 and
optimized_oracle_me_outputs_match_paper_exact.rs)."""
import numpy as np
import pytest

import oracle as O
from tests.helpers import ccs_case, ELL_D, D_SC, XS, kadd


@pytest.mark.parametrize("ell,k,inputs", [(4, 1, False), (4, 3, True), (5, 2, True), (3, 13, True)])
def test_round0_sum_is_hypercube_sum(ell, k, inputs):
    ccs, z, Z, ch, chals = ccs_case(ell, k, inputs)
    S = O.q_sum_hypercube(ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell)
    o = O.CcsOracle(ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell, D_SC)
    ys = o.evals_at(XS)
    assert np.array_equal(kadd(ys[0], ys[1]), S)
    if k == 1:
        assert np.all(S == 0)  # satisfied R1CS with in-range digits


@pytest.mark.parametrize("ell,k,inputs", [(4, 1, False), (4, 3, True), (5, 2, True), (3, 13, True)])
def test_final_running_sum_is_q_at_challenges(ell, k, inputs):
    ccs, z, Z, ch, chals = ccs_case(ell, k, inputs)
    S = O.q_sum_hypercube(ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell)
    o = O.CcsOracle(ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell, D_SC)
    rc, ev, fin = o.sumcheck_fixed(S, chals)
    assert rc == 0
    q = O.q_eval_ext(ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell,
                     chals[ell:], chals[:ell])
    assert np.array_equal(fin, q)
    y, ysc = o.me_outputs()
    for i in range(k):
        y2, ys2 = O.me_y_at_r(ccs, Z[i], ell, chals[:ell])
        assert np.array_equal(y[i], y2) and np.array_equal(ysc[i], ys2)


def test_invalid_witness_trips_invariant():
    ccs, z, Z, ch, chals = ccs_case(4, 1, False)
    z = z.copy()
    z[5] = (int(z[5]) + 1) % ((1 << 64) - (1 << 32) + 1)
    Zbad = O.decomp_b2(z)[None]
    o = O.CcsOracle(ccs, Zbad, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], None, ELL_D, 4, D_SC)
    rc, _, _ = o.sumcheck_fixed(np.zeros(2, np.uint64), chals)
    assert rc == -1  # round 0: p(0) + p(1) != claimed 0
