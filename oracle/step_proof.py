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
    # shout_addr_pre: ShoutAddrPreProof, empty without Shout instances
    s = rec.get("shout")
    if s is not None:
        W.kvec(s["sums"])
        W.u(s["active"])
        W.polys(s["polys"])
        W.kvec(s["r_addr"])
    else:
        W.w += [0, 0, 0, 0]
    # proofs: Vec<MemOrLutProof> (memory.rs:1555-1569), Shout entries first;
    # enum tags in declaration order, Twist = 0, Shout = 1
    n_lut = len(s["sums"]) if s is not None else 0
    W.u(n_lut + len(rec["twist"]))
    for _ in range(n_lut):
        W.w += [1, 0, 0, 0]  # ShoutProof { addr_pre: BatchedAddrProof::default() }
    v = rec.get("val_eval")
    per = 3 if (v is not None and v.get("has_prev")) else 2
    for i, tp in enumerate(rec["twist"]):
        W.u(0)
        W.kvec([(0, 0), (0, 0)])  # addr_pre: claimed sums (zero), read / write rounds, r_addr
        W.polys(tp["polys"])
        W.kvec(tp["r_addr"])
        base = per * i
        if v is None or base + per > len(v["sums"]):
            W.u(0)
            continue
        W.u(1)  # val_eval: Some(TwistValEvalProof)
        for c in range(per):
            if c == 2:
                W.u(1)
            W.k(v["sums"][base + c])
            if c == 2:
                W.u(1)
            W.u(len(v["polys"][base + c]))
            for rd in v["polys"][base + c]:
                W.kvec(rd)
        if per == 2:
            W.w += [0, 0]
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
    sums, active, polys, r_addr = R.kvec(), R.u(), R.polys(), R.kvec()
    f["shout"] = dict(sums=sums, active=active, polys=polys, r_addr=r_addr) if sums else None
    if not sums and (active or polys or r_addr):
        raise ValueError("shout_addr_pre must be empty when there are no Shout instances")
    f["twist"] = []
    vsums, vpolys, has_prev, n_ve = [], [], None, 0
    for _ in range(R.u()):
        tag = R.u()
        cs, pol, ra = R.kvec(), R.polys(), R.kvec()
        if tag == 1:
            if f["twist"] or cs or pol or ra:
                raise ValueError("a Shout proof entry must be empty and precede the Twist entries")
            continue
        if tag != 0:
            raise ValueError(f"unknown MemOrLutProof tag {tag}")
        if cs != [(0, 0), (0, 0)] or len(pol) != 2:
            raise ValueError("Twist addr_pre must carry two zero claimed sums and two claims")
        f["twist"].append(dict(polys=pol, r_addr=ra))
        if R.u():
            n_ve += 1
            for c in range(3):
                if c == 2:
                    prev = R.u()
                    if has_prev is None:
                        has_prev = bool(prev)
                    if bool(prev) != has_prev:
                        raise ValueError("rollover claims on some Twist instances only")
                    if not prev:
                        if R.u():
                            raise ValueError("rounds_prev_total without claimed_prev_inc_sum_total")
                        break
                vsums.append(R.k())
                if c == 2 and not R.u():
                    raise ValueError("claimed_prev_inc_sum_total without rounds_prev_total")
                vpolys.append([R.kvec() for _ in range(R.u())])
    if n_ve not in (0, len(f["twist"])):
        raise ValueError("val_eval on some Twist instances only")
    f["val_eval"] = dict(sums=vsums, polys=vpolys, has_prev=bool(has_prev)) if n_ve else None
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
    by a struct-order step proof, less the words the verifier derives itself
    (Twist address finals, r_val), which the struct does not hold.  A lane that
    mixes one instance has rho = I; its sampled coefficients are not part of the
    struct, and zeros stand in for them (the verifier then accepts any sampled
    value, as it uses rho = I).  verify_step(..., _struct=True) reads this."""
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
    for tp in f["twist"]:  # the address finals are not in the struct: the verifier derives them
        P += _round_major(tp["polys"], len(tp["r_addr"]))
        for v in tp["r_addr"]:
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
        P += _round_major(v["polys"], ell_n)  # r_val is transcript-derived, not in the struct
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
