"""StepProof in struct order (crates/neo-fold/src/shard_proof_types.rs:45-131)
as the canonical word dump that neo_gpu_shard_step_proof emits: every Vec
prefixed by its length, K = (re, im), F and integers one word, [u8; 32]
digests four little-endian words, byte strings a length then 8 bytes per word,
Option a 0 / 1 word then the value.

TEST INFRASTRUCTURE ONLY (the verifier restatement's reader and writer of that
layout); the product emits it from its own records (fold.cu).
"""
import numpy as np

from .fold import D, Q, rot_int


class Writer:
    def __init__(self):
        self.w = []

    def u(self, v):
        self.w.append(int(v) % (1 << 64))

    def k(self, v):
        self.w += [int(v[0]), int(v[1])]

    def fvec(self, v):
        self.u(len(v))
        self.w += [int(x) % Q for x in v]

    def kvec(self, v):
        self.u(len(v))
        for x in v:
            self.k(x)

    def digest(self, d):
        d = bytes(d)
        for i in range(4):
            self.u(int.from_bytes(d[8 * i:8 * i + 8], "little"))

    def bytes_(self, b):
        b = bytes(b)
        self.u(len(b))
        for i in range(0, len(b), 8):
            self.u(int.from_bytes(b[i:i + 8], "little"))

    def me(self, me, kappa, d_pad):
        """MeInstance: c, X, r, y, y_scalars, m_in, fold_digest, c_step_coords, u_offset, u_len."""
        self.u(D)
        self.u(kappa)
        self.fvec(me["c"])
        self.u(D)
        self.u(me["m_in"])
        self.fvec(me["X"])
        self.kvec(me["r"])
        self.u(len(me["y"]))
        for row in me["y"]:
            assert len(row) == d_pad
            self.kvec(row)
        self.kvec(me["ysc"])
        self.u(me["m_in"])
        self.digest(me["digest"])
        self.u(0)
        self.u(0)
        self.u(0)

    def mes(self, v, kappa, d_pad):
        self.u(len(v))
        for me in v:
            self.me(me, kappa, d_pad)

    def rhos(self, rhos):
        """Vec<Mat<F>>: rho_i = rot(a_i), the identity when one instance is mixed."""
        k = len(rhos)
        self.u(k)
        for a in rhos:
            R = np.eye(D, dtype=np.int64) if k == 1 else rot_int(np.array(a, np.int64))
            self.u(D)
            self.u(D)
            self.fvec([int(v) % Q for v in R.reshape(-1)])

    def polys(self, polys):
        self.u(len(polys))
        for claim in polys:
            self.u(len(claim))
            for rd in claim:
                self.kvec(rd)

    def lane(self, lane, kappa, d_pad):
        self.rhos(lane["rhos"])
        self.me(lane["parent"], kappa, d_pad)
        self.mes(lane["children"], kappa, d_pad)


def write_step(rec, kappa, d_pad):
    """The struct-order words of one verified step record (see OracleVerifier.verify_step)."""
    W = Writer()
    W.mes(rec["ccs_out"], kappa, d_pad)
    W.u(len(rec["ajtai_polys"]))
    for co in rec["ajtai_polys"]:
        W.kvec(co)
    W.u(1)
    W.k(rec["T"])
    W.kvec(list(rec["r_time"]) + list(rec["alpha_p"]))
    W.kvec(rec["alpha"])
    W.kvec(rec["beta_a"])
    W.kvec(rec["beta_r"])
    W.k(rec["gamma"])
    W.k(rec["final"])
    W.u(0)
    W.u(0)
    W.lane(rec["main"], kappa, d_pad)
    W.mes(rec["cpu_me_val"], kappa, d_pad)
    if rec.get("shout") is not None:
        s = rec["shout"]
        W.u(1)
        W.kvec(s["sums"])
        W.u(s["active"])
        W.polys(s["polys"])
        W.kvec(s["r_addr"])
    else:
        W.u(0)
    W.u(len(rec["twist"]))
    for tp in rec["twist"]:
        W.u(0)
        W.polys(tp["polys"])
        W.kvec(tp["r_addr"])
        W.kvec(tp["finals"])
    if rec.get("val_eval") is not None:
        v = rec["val_eval"]
        W.u(1)
        W.kvec(v["sums"])
        W.polys(v["polys"])
        W.kvec(v["r_val"])
    else:
        W.u(0)
    t = rec["time"]
    W.kvec(t["sums"])
    W.u(len(t["degs"]))
    for d in t["degs"]:
        W.u(d)
    W.u(len(t["labels"]))
    for lab in t["labels"]:
        W.bytes_(lab)
    W.polys(t["polys"])
    if rec.get("val") is not None:
        W.u(1)
        W.lane(rec["val"], kappa, d_pad)
    else:
        W.u(0)
    return np.array(W.w, dtype=np.uint64)


class Reader:
    def __init__(self, S):
        self.S = [int(v) for v in np.asarray(S, np.uint64).reshape(-1)]
        self.i = 0

    def u(self):
        if self.i >= len(self.S):
            raise ValueError("struct-order proof too short")
        v = self.S[self.i]
        self.i += 1
        return v

    def k(self):
        return (self.u(), self.u())

    def fvec(self):
        n = self.u()
        return [self.u() for _ in range(n)]

    def kvec(self):
        n = self.u()
        return [self.k() for _ in range(n)]

    def digest(self):
        return b"".join(self.u().to_bytes(8, "little") for _ in range(4))

    def bytes_(self):
        n = self.u()
        raw = b"".join(self.u().to_bytes(8, "little") for _ in range((n + 7) // 8))
        return raw[:n]

    def me(self):
        d, kappa = self.u(), self.u()
        c = self.fvec()
        rows, m_in = self.u(), self.u()
        X = self.fvec()
        r = self.kvec()
        y = [self.kvec() for _ in range(self.u())]
        ysc = self.kvec()
        m_in2 = self.u()
        dig = self.digest()
        coords = self.fvec()
        u_off, u_len = self.u(), self.u()
        return dict(c=c, X=X, r=r, y=y, ysc=ysc, m_in=m_in2, digest=dig, d=d, kappa=kappa, rows=rows,
                    cols=m_in, coords=coords, u_offset=u_off, u_len=u_len)

    def mes(self):
        return [self.me() for _ in range(self.u())]

    def rhos(self):
        out = []
        for _ in range(self.u()):
            rows, cols = self.u(), self.u()
            out.append(np.array(self.fvec(), dtype=np.uint64).reshape(rows, cols))
        return out

    def polys(self):
        return [[self.kvec() for _ in range(self.u())] for _ in range(self.u())]

    def lane(self):
        return dict(rhos=self.rhos(), parent=self.me(), children=self.mes())

    def done(self):
        if self.i != len(self.S):
            raise ValueError(f"{len(self.S) - self.i} struct-order words left over")


def read_step(S):
    """Fields of a struct-order step proof."""
    R = Reader(S)
    f = dict(ccs_out=R.mes())
    f["ajtai_polys"] = [R.kvec() for _ in range(R.u())]
    f["T"] = R.k() if R.u() else None
    f["chals"] = R.kvec()
    f["alpha"], f["beta_a"], f["beta_r"], f["gamma"] = R.kvec(), R.kvec(), R.kvec(), R.k()
    f["final"] = R.k()
    f["header_digest"] = R.fvec()
    f["extra"] = R.u()
    f["main"] = R.lane()
    f["cpu_me_val"] = R.mes()
    f["shout"] = dict(sums=R.kvec(), active=R.u(), polys=R.polys(), r_addr=R.kvec()) if R.u() else None
    f["twist"] = []
    for _ in range(R.u()):
        tag = R.u()
        f["twist"].append(dict(tag=tag, polys=R.polys(), r_addr=R.kvec(), finals=R.kvec()))
    f["val_eval"] = dict(sums=R.kvec(), polys=R.polys(), r_val=R.kvec()) if R.u() else None
    sums = R.kvec()
    degs = [R.u() for _ in range(R.u())]
    labels = [R.bytes_() for _ in range(R.u())]
    f["time"] = dict(sums=sums, degs=degs, labels=labels, polys=R.polys())
    f["val"] = R.lane() if R.u() else None
    R.done()
    return f


def _round_major(polys, n_rounds):
    """[claim][round][coeff] -> the transcript order: per round, per claim."""
    out = []
    for rd in range(n_rounds):
        for claim in polys:
            for c in claim[rd]:
                out += [c[0], c[1]]
    return out


def to_transcript_order(f, t, nb, ell_n):
    """The transcript-order proof words (neo_gpu_shard_fold_step's dump) carried
    by a struct-order step proof.  A lane that mixes one instance has rho = I;
    its sampled coefficients are not part of the struct, and zeros stand in for
    them (the verifier then accepts any sampled value, as it uses rho = I)."""
    P = []
    k = len(f["ccs_out"])
    P += list(f["ccs_out"][0]["c"])
    P += list(f["T"])
    if f["shout"] is not None:
        s = f["shout"]
        for v in s["sums"]:
            P += list(v)
        P.append(s["active"])
        P += _round_major(s["polys"], len(s["r_addr"]) if s["polys"] else 0)
        for v in s["r_addr"]:
            P += list(v)
    for tp in f["twist"]:
        P += _round_major(tp["polys"], len(tp["r_addr"]))
        for v in tp["r_addr"] + tp["finals"]:
            P += list(v)
    P += _round_major(f["time"]["polys"], ell_n)
    for co in f["ajtai_polys"]:
        for c in co:
            P += list(c)
    P += list(f["final"])
    for me in f["ccs_out"]:
        for j in range(t):
            for c in me["y"][j][:D]:
                P += list(c)
    for me in f["ccs_out"]:
        for j in range(t):
            P += list(me["ysc"][j])
    if nb:
        for me in f["ccs_out"]:
            for j in range(t, t + nb):
                for c in me["y"][j][:D]:
                    P += list(c)
            for j in range(t, t + nb):
                P += list(me["ysc"][j])
    if f["val_eval"] is not None:
        v = f["val_eval"]
        for x in v["sums"]:
            P += list(x)
        P += _round_major(v["polys"], ell_n)
        for x in v["r_val"]:
            P += list(x)
        for me in f["cpu_me_val"]:
            for j in range(t + nb):
                for c in me["y"][j][:D]:
                    P += list(c)
            for x in me["ysc"]:
                P += list(x)

    def lane(L):
        out = []
        kk = len(L["rhos"])
        for R in L["rhos"]:
            out += [0] * D if kk == 1 else [int(v) for v in R[:, 0]]  # column 0 of rot(a) is a
        for c in L["parent"]["c"]:
            out.append(c)
        for ch in L["children"]:
            out += list(ch["c"])
            for j in range(t + nb):
                for c in ch["y"][j][:D]:
                    out += list(c)
        return out

    P += lane(f["main"])
    if f["val"] is not None:
        P += lane(f["val"])
    return np.array([int(v) % (1 << 64) for v in P], dtype=np.uint64), k
