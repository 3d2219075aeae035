"""The benchmarked workloads checked word for word against the oracle.

* The single shard with memory exactly as bench.py builds it (n = m = 2^16,
  1024 trace steps per fold step, a Twist memory of 2^12 cells, a Shout table
  of 2^16 entries, the same seeds and PP): step 0 and two steady-state steps
  (k = 13) with the Twist rollover between chunks give the oracle's proof
  words and transcript state.
* The large shard (n = m = 2^20, a Twist memory of 2^16 cells, a Shout table
  of 2^20 entries) where the oracle is affordable: the MCS commitment of its
  witness under a setup_par PP, a two-plane commitment, the ME evaluations of
  the witness at a random point, and the first Pi_CCS row rounds at 2^20 rows.
"""
import types

import numpy as np
import pytest

import oracle as O
from oracle.fold import OracleShard
from nightstream_b200 import gpu, synth

Q = (1 << 64) - (1 << 32) + 1
pytestmark = pytest.mark.gpu


def test_bench_workload_steps_match_oracle(ctx):
    import bench
    args = types.SimpleNamespace(ell=16, chunk=1024, workload="memory")
    wl = bench.Workload(args, 0, 3)
    ctx.pp_upload(wl.pp)
    g = gpu.Shard(ctx, wl.ccs, m_in=1, k_rho=12, app_label=b"neo/bench", mem=wl.mem)
    o = OracleShard(wl.ccs, wl.pp, m_in=1, k_rho=12, app_label=b"neo/bench", mem=wl.mem)
    for c in range(3):
        wl.prepare(g, c)
        wl.prepare(o, c)
        pg = g.fold_step(wl.z(c))
        po = o.fold_step(wl.z(c))
        assert pg.shape == po.shape, f"step {c}: proof length {pg.shape} vs {po.shape}"
        assert np.array_equal(pg, po), f"step {c}: first mismatch at word {int(np.argmax(pg != po))}"
        assert np.array_equal(g.transcript_state(), o.tr.state()), f"step {c}: transcript state"
    g.close()


@pytest.fixture(scope="module")
def large():
    ccs, zs, mem, inits = synth.make_memory_workload_chunks(20, 4321, 1, 1 << 14, 20, 16)
    return ccs, zs[0]


def test_large_shard_commitments_match_oracle(ctx, large):
    ccs, z = large
    m = 1 << 20
    seed = bytes(range(3, 35))
    ctx.pp_generate(seed, 16, m, 1)
    pp = O.pp_setup(seed, 16, m, 1)
    Z0 = O.decomp_b2(z)
    assert np.array_equal(ctx.decomp_b2(z), Z0)
    assert np.array_equal(ctx.commit(Z0), O.commit_digits(pp, Z0))
    rng = np.random.default_rng(20)
    Z2 = rng.integers(-1, 2, size=(2, 54, m)).astype(np.int8)
    assert np.array_equal(ctx.commit(Z2), np.stack([O.commit_digits(pp, Z2[i]) for i in range(2)]))
    del pp


def test_large_shard_me_y_matches_oracle(ctx, large):
    ccs, z = large
    rng = np.random.default_rng(21)
    r = synth.uniform_k(rng, 20)
    Z0 = O.decomp_b2(z)
    y, ys = ctx.me_y(ccs, Z0, r)
    y2, ys2 = O.me_y_at_r(ccs, Z0, 20, r)
    assert np.array_equal(np.asarray(y).reshape(np.asarray(y2).shape), y2)
    assert np.array_equal(np.asarray(ys).reshape(np.asarray(ys2).shape), ys2)


def test_large_shard_first_row_rounds_match_oracle(ctx, large):
    """Pi_CCS at 2^20 rows with the MCS witness and four ternary children
    (270 digit rows: the pattern histogram takes two q chunks per block
    column there): rounds 0..5 (histogram, lookup-table and K-table kernels)."""
    ccs, z = large
    ell, k, ell_d, d_sc = 20, 5, 6, 6
    rng = np.random.default_rng(22)
    Z = np.stack([O.decomp_b2(z)] + [rng.integers(-1, 2, size=(54, 1 << ell)).astype(np.int8) for _ in range(k - 1)])
    uk = lambda n: synth.uniform_k(rng, n)
    args = (ccs, Z, 2, uk(ell_d), uk(ell_d), uk(ell), uk(1)[0], uk(ell), ell_d, ell, d_sc)
    g = gpu.GpuCcsOracle(ctx, *args)
    o = O.CcsOracle(*args)
    xs = np.array([[i, 0] for i in range(d_sc + 1)], np.uint64)
    chals = uk(6)
    for r in range(6):
        assert np.array_equal(g.evals_at(xs), o.evals_at(xs)), f"round {r}"
        g.fold(chals[r])
        o.fold(chals[r])
    g.close()
