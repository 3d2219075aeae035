"""The library's host transcript (C++) against the oracle's restatement (C):
identical sponge states through every operation kind; CCS digest equal.
Both restate crates/neo-transcript/src/poseidon2.rs; constants are unpinned."""
import numpy as np

import oracle as O
from nightstream_b200 import gpu, synth


def _drive(tr):
    out = []
    tr.append_message(b"lbl", b"hello")
    tr.append_fields(b"f", [1, 2, 3, 4, 5, 6, 7])
    tr.append_u64s(b"u", [(1 << 64) - 1, 5])
    out.append(tr.challenge_field(b"c0"))
    out += [int(v) for v in tr.challenge_fields(b"chal/k", 6)]
    out += list(tr.digest32())
    tr.append_fields(b"empty", [])
    tr.append_message(b"", b"")
    out.append(tr.challenge_field(b"c1"))
    out += [int(v) for v in tr.state()]
    return out


def test_transcript_matches_oracle():
    a = _drive(gpu.HostTranscript(b"neo/test"))
    b = _drive(O.Transcript(b"neo/test"))
    assert a == b


def test_transcript_distinct_labels_give_distinct_challenges():
    # crates/neo-transcript/tests/challenges.rs: label domain separation
    t1, t2 = gpu.HostTranscript(b"app"), gpu.HostTranscript(b"app")
    assert t1.challenge_field(b"a") != t2.challenge_field(b"b")


def test_ccs_digest_matches_oracle():
    ccs, _ = synth.make_r1cs(6, 3)
    assert np.array_equal(gpu.ccs_digest(ccs), O.ccs_digest(ccs))


def test_ccs_digest_cache_returns_each_ccs_its_own_digest():
    """The library keeps digests of CCSs it has seen (matched on an exact copy
    of the matrices): repeated and interleaved lookups, and a CCS that differs
    from a cached one in a single coefficient, all equal the oracle."""
    import copy
    from nightstream_b200 import synth
    a, _ = synth.make_r1cs(9, 41)
    b, _ = synth.make_r1cs(9, 42)
    c = copy.deepcopy(a)
    M = c.matrices[2]
    M.vals = M.vals.copy()
    M.vals[3] = (int(M.vals[3]) + 1) % ((1 << 64) - (1 << 32) + 1)
    want = {k: O.ccs_digest(x) for k, x in (("a", a), ("b", b), ("c", c))}
    for k, x in (("a", a), ("b", b), ("a", a), ("c", c), ("b", b), ("c", c), ("a", a)):
        assert np.array_equal(gpu.ccs_digest(x), want[k]), k
    assert not np.array_equal(want["a"], want["c"])


def test_ccs_digest_simd_and_scalar_paths_match_oracle():
    """The width-16 permutation behind the CCS digest has an AVX-512 path
    (taken when the host has AVX-512F) and a scalar one (NEO_TRANSCRIPT_SCALAR
    set): both give the oracle's digest, for a CCS whose digest takes some
    ten thousand permutations."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path.insert(0, %r); from nightstream_b200 import gpu, synth; "
            "ccs, _ = synth.make_r1cs(12, 17); print(','.join(str(int(v)) for v in gpu.ccs_digest(ccs)))" % root)
    ccs, _ = synth.make_r1cs(12, 17)
    want = ",".join(str(int(v)) for v in O.ccs_digest(ccs))
    for extra in ({}, {"NEO_TRANSCRIPT_SCALAR": "1"}):
        env = {k: v for k, v in os.environ.items() if k != "NEO_TRANSCRIPT_SCALAR"}
        env.update(extra)
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
        assert out.stdout.strip() == want, extra


def _drive_many(tr):
    """3000 absorbs of 23 random, edge-value (q - 1 - small) or small field
    elements with a challenge every 50: about 20 k permutations."""
    q = (1 << 64) - (1 << 32) + 1
    rng = np.random.default_rng(11)
    out = []
    for i in range(3000):
        kind = i % 3
        if kind == 0:
            vals = [int(v) for v in rng.integers(0, q, size=23, dtype=np.uint64)]
        elif kind == 1:
            vals = [q - 1 - int(v) for v in rng.integers(0, 4, size=23)]
        else:
            vals = [int(v) for v in rng.integers(0, 16, size=23)]
        tr.append_fields(b"y_elem", vals)
        if i % 50 == 0:
            out.append(int(tr.challenge_field(b"chal")))
    return out + [int(v) for v in tr.state()]


def test_transcript_simd_and_scalar_paths_match_oracle():
    """The width-8 transcript permutation has an AVX-512 path (lanes 1..7 of
    the partial rounds in one vector; taken when the host has AVX-512F) and a
    scalar one (NEO_TRANSCRIPT_SCALAR set): both follow the oracle's sponge
    through about twenty thousand permutations of random, edge-value and
    small-value absorbs."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

    code = ("import sys; sys.path.insert(0, %r); sys.path.insert(0, %r); import test_transcript as T; "
            "from nightstream_b200 import gpu; print(','.join(map(str, T._drive_many(gpu.HostTranscript(b'neo/simd')))))"
            % (root, os.path.join(root, "tests")))
    want = ",".join(map(str, _drive_many(O.Transcript(b"neo/simd"))))
    for extra in ({}, {"NEO_TRANSCRIPT_SCALAR": "1"}):
        env = {k: v for k, v in os.environ.items() if k != "NEO_TRANSCRIPT_SCALAR"}
        env.update(extra)
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
        assert out.stdout.strip() == want, extra
