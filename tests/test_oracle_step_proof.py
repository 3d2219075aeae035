"""StepProof in struct order (crates/neo-fold/src/shard_proof_types.rs:45-131,
the layout of neo_gpu_shard_step_proof): the verifier restatement writes it
while it replays a step, reads it back, verifies the step from it, and rejects
a struct whose derived fields (ME claims, the RLC parent, digests, public
challenges) differ from its own replay."""
import numpy as np
import pytest

from nightstream_b200 import synth
from oracle.fold import OracleShard
from oracle.step_proof import read_step, to_transcript_order, write_step
from oracle.verify import OracleVerifier, VerifyError

Q = (1 << 64) - (1 << 32) + 1


def _case(memory):
    if memory:
        ccs, zs, mem, inits = synth.make_memory_workload_chunks(10, 3, 3, 16, 6, 5)
    else:
        ccs, z = synth.make_r1cs(9, 8)
        zs, mem, inits = [z] * 3, None, None
    pp = np.random.default_rng(4).integers(0, Q, size=(16, ccs.m, 54), dtype=np.uint64)
    sh = OracleShard(ccs, pp, m_in=1, k_rho=12, app_label=b"neo/struct", mem=mem)
    v = OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/struct", mem=mem)
    out = []
    for c in range(3):
        if c and inits:
            sh.set_twist_init(0, inits[c][0])
            v.set_twist_init(0, inits[c][0])
        P = sh.fold_step(zs[c])
        rec = {}
        assert v.verify_step(zs[c][:1], P, record=rec)
        out.append((zs[c], P, write_step(rec, 16, 64)))
    return ccs, mem, inits, out


@pytest.fixture(scope="module", params=[False, True], ids=["main", "memory"])
def steps(request):
    return _case(request.param)


def _fresh(ccs, mem):
    return OracleVerifier(ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/struct", mem=mem)


def test_struct_round_trip_and_verify(steps):
    ccs, mem, inits, out = steps
    v = _fresh(ccs, mem)
    for c, (z, P, S) in enumerate(out):
        f = read_step(S)
        assert len(f["ccs_out"]) == (1 if c == 0 else 13) and len(f["main"]["children"]) == 12
        P2, k = to_transcript_order(f, ccs.t, v.bus.bus_cols, v.ell_n)
        # words the verifier derives are not in the struct: per Twist instance
        # its two address finals, and r_val of the val-eval batch
        derived = 4 * len(f["twist"]) + (2 * v.ell_n if f["val_eval"] is not None else 0)
        assert len(P2) == len(P) - derived
        if k > 1 and not derived:  # (a one-instance lane's sampled rho is not in the struct either)
            assert np.array_equal(P2, np.asarray(P, np.uint64))
        if c and inits:
            v.set_twist_init(0, inits[c][0])
        assert v.verify_step_struct(z[:1], S)


def test_struct_rejects_changed_derived_fields(steps):
    """Words the transcript-order proof does not carry (r of the ME claims, the
    RLC parent's X, a child's fold digest, a public challenge) are checked
    against the replay."""
    ccs, mem, inits, out = steps
    z, P, S = out[1]
    f = read_step(S)
    n = len(S)
    # locate a few derived words by re-serialising with one field changed
    for mutate in ("r", "parent_X", "digest", "beta"):
        g = read_step(S)
        if mutate == "r":
            g["ccs_out"][0]["r"][0] = ((g["ccs_out"][0]["r"][0][0] + 1) % Q, g["ccs_out"][0]["r"][0][1])
        elif mutate == "parent_X":
            g["main"]["parent"]["X"][0] = (g["main"]["parent"]["X"][0] + 1) % Q
        elif mutate == "digest":
            d = bytearray(g["main"]["children"][3]["digest"])
            d[0] ^= 1
            g["main"]["children"][3]["digest"] = bytes(d)
        else:
            g["beta_r"][0] = ((g["beta_r"][0][0] + 1) % Q, g["beta_r"][0][1])
        S_bad = _rewrite(g)
        assert len(S_bad) == n and not np.array_equal(S_bad, S)
        v = _fresh(ccs, mem)
        assert v.verify_step_struct(out[0][0][:1], out[0][2])
        if inits:
            v.set_twist_init(0, inits[1][0])
        with pytest.raises(VerifyError):
            v.verify_step_struct(z[:1], S_bad)


def test_struct_memory_fields(steps):
    """The memory sidecar in MemSidecarProof order: Shout entries (empty
    BatchedAddrProof) before one Twist entry per instance, each with zero
    address claimed sums, read / write rounds, r_addr and its val-eval claims
    (lt, total and, from the second step on, the rollover total)."""
    ccs, mem, inits, out = steps
    for c, (z, P, S) in enumerate(out):
        f = read_step(S)
        if mem is None:
            assert f["shout"] is None and f["twist"] == [] and f["val_eval"] is None
            continue
        assert len(f["twist"]) == len(mem["twist"])
        for tp in f["twist"]:
            assert len(tp["polys"]) == 2 and all(len(cl) == len(tp["r_addr"]) for cl in tp["polys"])
        ve = f["val_eval"]
        assert ve is not None and ve["has_prev"] == (c > 0)
        assert len(ve["sums"]) == (3 if c else 2) * len(mem["twist"]) == len(ve["polys"])


def _rewrite(f):
    """Struct-order words of parsed fields (the inverse of read_step)."""
    rec = dict(ccs_out=f["ccs_out"], ajtai_polys=f["ajtai_polys"], T=f["T"],
               r_time=f["chals"][:len(f["ccs_out"][0]["r"])], alpha_p=f["chals"][len(f["ccs_out"][0]["r"]):],
               alpha=f["alpha"], beta_a=f["beta_a"], beta_r=f["beta_r"], gamma=f["gamma"], final=f["final"],
               main=_lane_rec(f["main"]), cpu_me_val=f["cpu_me_val"], shout=f["shout"], twist=f["twist"],
               val_eval=f["val_eval"], time=f["time"], val=_lane_rec(f["val"]) if f["val"] else None)
    return write_step(rec, 16, 64)


def _lane_rec(L):
    k = len(L["rhos"])
    rhos = [[0] * 54] if k == 1 else [[(int(v) if int(v) < Q // 2 else int(v) - Q) for v in R[:, 0]] for R in L["rhos"]]
    return dict(rhos=rhos, parent=L["parent"], children=L["children"])


def test_struct_rejects_malformed_words(steps):
    ccs, mem, inits, out = steps
    v = _fresh(ccs, mem)
    with pytest.raises(VerifyError):
        v.verify_step_struct(out[0][0][:1], np.asarray(out[0][2], np.uint64)[:-3])
