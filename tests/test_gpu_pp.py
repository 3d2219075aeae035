"""Ajtai PP generated on the device (neo_gpu_pp_generate, neo_gpu_chacha8_sample)
against the C oracle: bit-exact (crates/neo-ajtai/src/commit.rs:21-264)."""
import time

import numpy as np
import pytest

import oracle as O
from nightstream_b200 import gpu
from tests.pyref import pp_par_streams

Q = (1 << 64) - (1 << 32) + 1
pytestmark = pytest.mark.gpu
SEED = bytes((11 * i + 5) & 0xFF for i in range(32))


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("kappa,m", [(16, 1000), (3, 100), (4, 40000), (16, 1001), (16, 4096)])
def test_pp_generate_matches_oracle(ctx, mode, kappa, m):
    ctx.pp_generate(SEED, kappa, m, mode)
    got = ctx.pp_download(m, kappa)
    assert np.array_equal(got, O.pp_setup(SEED, kappa, m, mode))


@pytest.mark.parametrize("bound", [Q, (1 << 64) - (1 << 58), 1 << 63, 3 << 62])
def test_chacha8_sample_rejection_paths(ctx, bound):
    seeds = [bytes((i * 37 + j) & 0xFF for j in range(32)) for i in range(6)]
    counts = [0, 1, 7, 5000, 20000, 2048]
    got = ctx.chacha8_sample(seeds, counts, bound)
    assert np.array_equal(got, O.chacha8_sample(seeds, counts, bound))
    assert int(got.max(initial=0)) < bound


def test_generated_pp_commits_like_materialized(ctx):
    """The seeded-PP relation (neo-ajtai tests/seeded_pp_commit_matches_materialized.rs):
    committing with the device-generated setup_par PP equals committing with the
    same PP materialized on the host."""
    m = 2000
    ctx.pp_generate(SEED, 16, m, 1)
    Z = np.random.default_rng(5).integers(-1, 2, size=(3, 54, m)).astype(np.int8)
    got = ctx.commit(Z)
    pp = O.pp_setup(SEED, 16, m, 1)
    for v in range(3):
        assert np.array_equal(got[v], O.commit_digits(pp, Z[v]))


def test_pp_generate_errors(ctx):
    with pytest.raises(gpu.NeoGpuError):
        ctx.pp_generate(SEED, 16, 1024, 7)
    with pytest.raises(gpu.NeoGpuError):
        ctx.pp_generate(SEED, 0, 1024, 1)
    with pytest.raises(ValueError):
        ctx.pp_generate(SEED[:16], 16, 1024, 1)
    ctx.pp_generate(SEED, 2, 1024, 1)
    with pytest.raises(gpu.NeoGpuError):
        ctx.pp_download(1024, 2, first=2 * 1024 * 54 - 3, count=4)


def test_pp_generate_setup_m16_whole(ctx):
    """setup (one sequential stream) at m = 2^16, kappa = 16: 56.6 M coefficients."""
    m = 1 << 16
    ctx.pp_generate(SEED, 16, m, 0)
    assert np.array_equal(ctx.pp_download(m, 16), O.pp_setup(SEED, 16, m, 0))


def test_pp_generate_full_size_setup_par(ctx):
    """m = 2^20, kappa = 16 (7.25 GB): the first and last chunk-stream prefixes
    of every row against the oracle's streams from the same chunk seeds."""
    m, kappa = 1 << 20, 16
    t0 = time.perf_counter()
    ctx.pp_generate(SEED, kappa, m, 1)
    dt = time.perf_counter() - t0
    streams = pp_par_streams(SEED, kappa, m)
    per_row = len(streams) // kappa
    n = 54 * 512
    for i in range(kappa):
        for c in (0, per_row - 1):
            seed, lo, cols = streams[i * per_row + c]
            ref = O.chacha8_sample([seed], [n], Q)
            got = ctx.pp_download(m, kappa, first=(i * m + lo) * 54, count=n)
            assert np.array_equal(got, ref), (i, c)
    print(f"pp_generate setup_par kappa=16 m=2^20: {dt * 1e3:.1f} ms (host seed derivation + device sampling)")
