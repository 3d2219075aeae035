"""Pins the oracle (and through it the library) to values exported from the
reference's own Rust crates by tests/golden/export (a cargo program to run
on a machine with crates.io access; see its Cargo.toml).  Until its output,
tests/golden/reference_vectors.json, is present these tests are skipped: the
Poseidon2 constants and the ChaCha8 streams come from un-vendored crates
(p3-poseidon2 / p3-goldilocks 0.4.1, rand_chacha 0.9.0), so nothing else in
this repository can pin them."""
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
VECTORS = os.path.join(HERE, "golden", "reference_vectors.json")
U64_MAX = (1 << 64) - 1


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(VECTORS):
        pytest.skip("tests/golden/reference_vectors.json not exported yet (needs cargo: tests/golden/export)")
    with open(VECTORS) as f:
        return json.load(f)


def _u64s(xs):
    return np.array([int(x) for x in xs], np.uint64)


def seed_from_u64(state):
    """rand_core 0.9 SeedableRng::seed_from_u64: a 32-byte seed from PCG32
    (XSH-RR) steps of the u64 state, 4 little-endian bytes per step."""
    out = b""
    mask = (1 << 64) - 1
    for _ in range(8):
        state = (state * 6364136223846793005 + 11634580027462260723) & mask
        xs = (((state >> 18) ^ state) >> 27) & 0xFFFFFFFF
        rot = state >> 59
        out += (((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF).to_bytes(4, "little")
    return out


def test_export_harness_is_committed():
    src = os.path.join(HERE, "golden", "export", "src", "main.rs")
    text = open(src).read()
    for key in ("poseidon2_w8_permute_0_to_7", "poseidon2_w16_permute_0_to_15", "pp_setup_par_row0_col0",
                "transcript_state_after_challenge"):
        assert key in text


def test_poseidon2_width8_matches_reference(ref):
    st = np.arange(8, dtype=np.uint64)
    O.lib().or_poseidon2_permute(O.ptr(st))
    assert np.array_equal(st, _u64s(ref["poseidon2_w8_permute_0_to_7"]))


def test_poseidon2_width16_matches_reference(ref):
    st = np.arange(16, dtype=np.uint64)
    O.lib().or_poseidon2_w16_permute(O.ptr(st))
    assert np.array_equal(st, _u64s(ref["poseidon2_w16_permute_0_to_15"]))


def test_chacha8_streams_match_reference(ref):
    seed8 = bytes(int(b) for b in ref["poseidon2_w8_seed"])
    got = O.chacha8_sample([seed8], [64], U64_MAX)
    assert np.array_equal(got, _u64s(ref["chacha8_from_seed_w8_seed_first_64"]))
    got = O.chacha8_sample([seed_from_u64(0x434353445F4D4154)], [64], U64_MAX)
    assert np.array_equal(got, _u64s(ref["chacha8_seed_from_u64_ccs_digest_first_64"]))


def test_setup_par_matches_reference(ref):
    seed = bytes(int(b) for b in ref["pp_seed"])
    kappa, m = int(ref["pp_kappa"]), int(ref["pp_m"])
    pp = O.pp_setup(seed, kappa, m, 1)
    assert np.array_equal(pp[0, 0], _u64s(ref["pp_setup_par_row0_col0"]))
    assert np.array_equal(pp[0, m - 1], _u64s(ref["pp_setup_par_row0_col_last"]))
    assert np.array_equal(pp[kappa - 1, 0], _u64s(ref["pp_setup_par_row_last_col0"]))


def test_transcript_matches_reference(ref):
    from nightstream_b200 import gpu
    label = ref["transcript_app_label"].encode()
    chal = ref["transcript_challenge_label"].encode()
    t = O.Transcript(label)
    assert np.array_equal(t.state(), _u64s(ref["transcript_state_after_new"]))
    assert t.challenge_field(chal) == int(ref["transcript_challenge"])
    assert np.array_equal(t.state(), _u64s(ref["transcript_state_after_challenge"]))
    lt = gpu.HostTranscript(label)  # the library's host transcript
    assert np.array_equal(lt.state(), _u64s(ref["transcript_state_after_new"]))
