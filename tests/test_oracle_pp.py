"""Ajtai PP generation on the CPU restatement (crates/neo-ajtai/src/commit.rs:21-264):
the C oracle's ChaCha8 and setup / setup_par partition against the independent
pure-Python restatement in pyref.py."""
import numpy as np
import pytest

import oracle
from pyref import ChaCha8, Q, pp_par_streams

SEED = bytes((7 * i + 3) & 0xFF for i in range(32))


def test_chacha8_stream_matches_python_restatement():
    raw = oracle.chacha8_sample([SEED], [300], (1 << 64) - 1)  # bound 2^64-1: no value of this stream is rejected
    c = ChaCha8(SEED)
    assert [int(v) for v in raw] == [c.next_u64() for _ in range(300)]


def test_bound_rejection_filters_the_stream():
    raw = oracle.chacha8_sample([SEED, SEED[::-1]], [8000, 40], (1 << 64) - 1)
    got = oracle.chacha8_sample([SEED, SEED[::-1]], [1000, 3], 1 << 62)
    a = raw[:8000]
    assert (a < (1 << 62)).sum() >= 1000
    assert np.array_equal(got[:1000], a[a < (1 << 62)][:1000])
    b = raw[8000:]
    assert np.array_equal(got[1000:], b[b < (1 << 62)][:3])


def test_setup_is_one_stream():
    pp = oracle.pp_setup(SEED, 3, 50, 0)
    assert pp.shape == (3, 50, 54)
    assert np.array_equal(pp.reshape(-1), oracle.chacha8_sample([SEED], [3 * 50 * 54], Q))
    assert int(pp.max()) < Q


@pytest.mark.parametrize("m", [100, 1024, 1500, (1 << 15) + 7])
def test_setup_par_partition(m):
    kappa = 2
    pp = oracle.pp_setup(SEED, kappa, m, 1)
    streams = pp_par_streams(SEED, kappa, m)
    ref = oracle.chacha8_sample([s for s, _, _ in streams], [n * 54 for _, _, n in streams], Q)
    assert np.array_equal(pp.reshape(-1), ref)
    # row 0 of setup_par differs from setup (the stream is partitioned)
    assert not np.array_equal(pp[0], oracle.pp_setup(SEED, kappa, m, 0)[0])


def test_chacha8_block_matches_published_vector():
    """ChaCha with 8 rounds, 256-bit all-zero key, zero nonce and counter: the
    first 64 keystream bytes of the published test vector TC1
    (draft-strombergson-chacha-test-vectors-01, 8 rounds).  rand_chacha's
    ChaCha8Rng::from_seed([0; 32]) returns these bytes as its first eight
    next_u64 values (little-endian), so this pins the block function, the key
    layout and the word order the PP sampler and the Poseidon2 constants use."""
    tc1 = bytes.fromhex(
        "3e00ef2f895f40d67f5bb8e81f09a5a12c840ec3ce9a7f3b181be188ef711a1e"
        "984ce172b9216f419f445367456d5619314a42a3da86b001387bfdb80e0cfe42")
    v = oracle.chacha8_sample([bytes(32)], [8], (1 << 64) - 1)
    assert b"".join(int(x).to_bytes(8, "little") for x in v) == tc1
