"""Verifier restatement of a Neo fold step, run on the canonical step-proof dump.

TEST INFRASTRUCTURE ONLY: it checks the proofs that neo_gpu_shard_fold_step
and oracle/fold.py emit.  It follows fold_shard_verify_impl
(crates/neo-fold/src/shard.rs:2482-2900) and verify_rlc_dec_lane
(shard.rs:1333-1420): it replays the Fiat-Shamir transcript from public data
and proof words only (no witness, no public parameters), checks every
sum-check round (p(0) + p(1) = running claim), the Pi_CCS terminal identity
rhs_terminal_identity_paper_exact
(neo-reductions/src/engines/optimized_engine/common.rs:702-836) against the
public initial sum claimed_initial_sum_from_inputs (common.rs:839-947), the
RLC mix of commitments / X / y (ccs::rlc_public) and the DEC reconstruction
(ccs::verify_dec_public), and carries the verified child ME claims to the
next step as the accumulator.
"""
import numpy as np

from . import Transcript, ccs_digest, decomp_b2, split_b
from .fold import D, Q, BusLayout, digest_fields, header_params, kadd, kmulp, le64, rot_int

ONE, ZERO = (1, 0), (0, 0)


class VerifyError(Exception):
    pass


def ksub(a, b):
    return ((a[0] - b[0]) % Q, (a[1] - b[1]) % Q)


def kpoly(co, x):
    """p(x) for coefficients low -> high."""
    acc = ZERO
    for c in reversed(co):
        acc = kadd(kmulp(acc, x), c)
    return acc


def keq(p, q):
    """eq_points (optimized_engine/common.rs:33-41)."""
    acc = ONE
    for a, b in zip(p, q):
        acc = kmulp(acc, kadd(kmulp(ksub(ONE, a), ksub(ONE, b)), kmulp(a, b)))
    return acc


def chi_table(pt):
    out = []
    for idx in range(1 << len(pt)):
        w = ONE
        for bit, a in enumerate(pt):
            w = kmulp(w, a if (idx >> bit) & 1 else ksub(ONE, a))
        out.append(w)
    return out


def kpow(x, e):
    acc = ONE
    for _ in range(e):
        acc = kmulp(acc, x)
    return acc


def centered(v):
    v = int(v) % Q
    return v - Q if v > Q // 2 else v


class Reader:
    """Cursor over the proof words of one step."""

    def __init__(self, P):
        self.P = [int(v) for v in np.asarray(P, np.uint64).reshape(-1)]
        self.i = 0

    def take(self, n):
        if self.i + n > len(self.P):
            raise VerifyError("proof too short")
        out = self.P[self.i:self.i + n]
        self.i += n
        return out

    def k(self):
        a, b = self.take(2)
        return (a, b)

    def ks(self, n):
        return [self.k() for _ in range(n)]

    def done(self):
        if self.i != len(self.P):
            raise VerifyError(f"{len(self.P) - self.i} proof words left over")


class OracleVerifier:
    """Public side of one shard: the CCS, m_in, k_rho, kappa, the application
    label and (for memory shards) the Shout tables / Twist initial states."""

    def __init__(self, ccs, m_in=1, k_rho=12, kappa=16, app_label=b"neo/shard", mem=None):
        self.ccs, self.m_in, self.k_rho, self.kappa, self.b = ccs, m_in, k_rho, kappa, 2
        self.n, self.m, self.t = ccs.n, ccs.m, ccs.t
        self.ell_n = (self.n - 1).bit_length()
        self.ell_d = 6
        self.d_sc = max(ccs.f_degree + 1, 2 * self.b + 2)
        self.lam, self.slack = header_params(self.ell_n + self.ell_d, self.d_sc)
        self.digest = ccs_digest(ccs)
        self.tr = Transcript(app_label)
        self.acc = []
        self.val_obligations = []
        self.step_idx = 0
        self.mem = mem or dict(steps=0, shout=[], twist=[])
        self.shout = [dict(sd) for sd in self.mem.get("shout", [])]
        self.twist = [dict(w) for w in self.mem.get("twist", [])]
        self.bus = BusLayout(self.m, m_in, self.mem.get("steps", 0), [s["ell_addr"] for s in self.shout],
                             [w["ell_addr"] for w in self.twist])
        self.shout_digest = [digest_fields(b"shout/table", [int(v) for v in s["table"]]) for s in self.shout]
        self.twist_digest = []
        for w in self.twist:
            init = w.get("init", [])
            if init:
                fs = []
                for a, v in init:
                    fs += [a, v]
                self.twist_digest.append(digest_fields(b"twist/init/sparse", fs))
            else:
                self.twist_digest.append(digest_fields(b"twist/init/zero", []))
        self.prev = None  # previous step's MCS commitment, X and Twist MemInits (rollover)

    # ---------------------------------------------------------------- transcript --
    def _k(self, label, v):
        self.tr.append_fields(label, np.array(v, np.uint64))

    def _chal(self, l0=b"batched/challenge/0", l1=b"batched/challenge/1"):
        return (int(self.tr.challenge_field(l0)), int(self.tr.challenge_field(l1)))

    def _sample_ext_point(self, label, l0, l1, n):
        out = []
        for i in range(n):
            self.tr.append_message(label, le64(i))
            out.append((int(self.tr.challenge_field(l0)), int(self.tr.challenge_field(l1))))
        return out

    def _batched(self, labels, degs, sums, n_rounds, R):
        """verify side of run_batched_sumcheck_prover (neo-reductions/src/sumcheck.rs:350-456)."""
        tr = self.tr
        running = list(sums)
        chals = []
        self.last_polys = [[] for _ in degs]  # [claim][round][coefficient]
        for rd in range(n_rounds):
            tr.append_message(b"batched/round_idx", le64(rd))
            polys = [R.ks(deg + 1) for deg in degs]
            for ci, co in enumerate(polys):
                self.last_polys[ci].append(co)
            for ci, (lab, co) in enumerate(zip(labels, polys)):
                p0, p1 = co[0], ZERO
                for c in co:
                    p1 = kadd(p1, c)
                if kadd(p0, p1) != running[ci]:
                    raise VerifyError(f"{lab.decode()} round {rd}: p(0) + p(1) != running claim")
                tr.append_message(b"batched/claim_label", lab)
                tr.append_message(b"batched/claim_idx", le64(ci))
                for c in co:
                    self._k(b"batched/round/coeff", c)
            r = self._chal()
            chals.append(r)
            running = [kpoly(co, r) for co in polys]
        return chals, running

    def _batched_ds(self, domain, inst_idx, labels, degs, sums, n_rounds, R):
        self.tr.append_message(b"sc/domain", domain)
        self.tr.append_message(b"sc/inst_idx", le64(inst_idx))
        out = self._batched(labels, degs, sums, n_rounds, R)
        self.tr.append_message(b"sc/domain_end", domain)
        self.tr.append_message(b"sc/inst_idx_end", le64(inst_idx))
        return out

    # ------------------------------------------------------------ ME helpers --
    def _yscalars(self, y):
        """y_scalars = sum_rho b^rho y[rho] per row."""
        out = []
        for row in y:
            acc, pw = ZERO, 1
            for rho in range(D):
                acc = kadd(acc, ((row[rho][0] * pw) % Q, (row[rho][1] * pw) % Q))
                pw = pw * self.b % Q
            out.append(acc)
        return out

    def _me(self, c, X, r, y_rows, digest):
        """ME claim with y rows padded to 2^ell_d and y_scalars derived from y."""
        d_pad = 1 << self.ell_d
        y = [list(row) + [ZERO] * (d_pad - len(row)) for row in y_rows]
        return dict(c=list(c), X=list(X), m_in=self.m_in, r=list(r), y=y, ysc=self._yscalars(y_rows),
                    digest=digest)

    def _initial_sum(self, alpha, gamma, k):
        """claimed_initial_sum_from_inputs (optimized_engine/common.rs:839-947), core rows."""
        if k < 2:
            return ZERO
        chi_a = chi_table(alpha)
        gk = kpow(gamma, k)
        inner, gkj = ZERO, ONE
        for j in range(self.t):
            gi = ONE
            for me in self.acc:
                gi = kmulp(gi, gamma)
                ye = ZERO
                for rho, w in enumerate(chi_a):
                    ye = kadd(ye, kmulp(me["y"][j][rho], w))
                inner = kadd(inner, kmulp(kmulp(gi, gkj), ye))
            gkj = kmulp(gkj, gk)
        return kmulp(gk, inner)

    def _terminal_rhs(self, alpha, beta_a, beta_r, gamma, r_prime, alpha_prime, y_out, r_in):
        """rhs_terminal_identity_paper_exact (optimized_engine/common.rs:702-836).
        y_out[i][j] = the 54 K entries of output i, matrix j."""
        k = len(y_out)
        eq_beta = kmulp(keq(alpha_prime, beta_a), keq(r_prime, beta_r))
        eq_ar = kmulp(keq(alpha_prime, alpha), keq(r_prime, r_in)) if r_in is not None else ZERO
        # F' from the first output's recomposed rows
        mvals = self._yscalars(y_out[0])
        fp = ZERO
        for coeff, exps in self.ccs.f_terms:
            term = ((coeff % Q), 0)
            for j, e in enumerate(exps):
                term = kmulp(term, kpow(mvals[j], e))
            fp = kadd(fp, term)
        chi_ap = chi_table(alpha_prime)

        def y_at(row):
            acc = ZERO
            for rho in range(D):
                acc = kadd(acc, kmulp(row[rho], chi_ap[rho]))
            return acc

        nc, g = ZERO, gamma
        for i in range(k):
            yv = y_at(y_out[i][0])
            prod = ONE
            for tt in range(-(self.b - 1), self.b):
                prod = kmulp(prod, ksub(yv, (tt % Q, 0)))
            nc = kadd(nc, kmulp(g, prod))
            g = kmulp(g, gamma)
        gk = kpow(gamma, k)
        ev = ZERO
        if r_in is not None and k >= 2:
            for j in range(self.t):
                for i in range(1, k):  # weight gamma^i (gamma^k)^j, i the 0-based output index
                    w = kmulp(kpow(gamma, i), kpow(gk, j))
                    ev = kadd(ev, kmulp(w, y_at(y_out[i][j])))
        return kadd(kmulp(eq_beta, kadd(fp, nc)), kmulp(eq_ar, kmulp(gk, ev)))

    # ---------------------------------------------------------- RLC / DEC lane --
    def _lane(self, lane, idx, ins, r, digest, R, rec=None):
        """verify_rlc_dec_lane (shard.rs:1333-1420): transcript binding, rho
        sampling, RLC public mix, DEC reconstruction; returns the children."""
        tr, t, kappa, m_in, nb = self.tr, self.t, self.kappa, self.m_in, self.bus.bus_cols
        k = len(ins)
        tr.append_message(b"fold/rlc_inputs/v1", lane)
        tr.append_u64s(b"step_idx", [idx])
        tr.append_u64s(b"me_count", [k])
        for me in ins:
            tr.append_fields(b"c_data", me["c"])
            tr.append_u64s(b"m_in", [me["m_in"]])
            tr.append_message(b"me_fold_digest", me["digest"])
            for rl in me["r"]:
                self._k(b"r_limb", rl)
            tr.append_fields(b"X", me["X"])
            for yj in me["y"]:
                for ye in yj:
                    self._k(b"y_elem", ye)
            for ysc in me["ysc"]:
                self._k(b"y_scalar", ysc)
            tr.append_u64s(b"c_step_coords_len", [0])
            tr.append_fields(b"c_step_coords", [])
            tr.append_u64s(b"u_offset", [0])
            tr.append_u64s(b"u_len", [0])
        # sample_rot_rhos_n (common.rs:467-573): must equal the proof's rhos
        A5 = [-2, -1, 0, 1, 2]
        bucket = (1 << 16) // 5 * 5
        rhos = np.zeros((k, D), np.int64)
        for i in range(k):
            tr.append_message(b"rlc/rot/index", le64(i))
            got, ctr = 0, i
            while got < D:
                tr.append_message(b"rlc/rot/chunk", le64(ctr))
                dig = tr.digest32()
                for w in range(16):
                    if got == D:
                        break
                    xv = dig[2 * w] | (dig[2 * w + 1] << 8)
                    if xv < bucket:
                        rhos[i, got] = A5[xv % 5]
                        got += 1
                ctr += 1
        proof_rhos = [centered(v) for v in R.take(k * D)]
        # a lane of one instance uses rho = I; the struct-order proof does not carry its sampled vector
        if not (k == 1 and getattr(self, "_struct", False)) and proof_rhos != [int(v) for v in rhos.reshape(-1)]:
            raise VerifyError(f"{lane.decode()} lane: RLC rho mismatch (transcript vs proof)")
        Rs = [np.eye(D, dtype=np.int64)] if k == 1 else [rot_int(rhos[i]) for i in range(k)]

        def mix(vecs):  # vecs[i]: list of 54-vectors of F_q ints -> sum_i rot(rho_i) vec, mod q
            acc_lo = acc_hi = 0
            for i in range(k):
                V = np.array(vecs[i], dtype=np.uint64).reshape(-1, D)
                lo = (V & np.uint64(0xFFFFFFFF)).astype(np.int64)
                hi = (V >> np.uint64(32)).astype(np.int64)
                acc_lo = acc_lo + lo @ Rs[i].T  # |entries| < 13 * 54 * 4 * 2^32 < 2^46
                acc_hi = acc_hi + hi @ Rs[i].T
            return [[(int(a) + (int(b) << 32)) % Q for a, b in zip(ra, rb)] for ra, rb in zip(acc_lo, acc_hi)]

        # RLC public mix (ccs::rlc_public): commitments, X, y (core and bus rows)
        c_parent = mix([[me["c"][c * D:(c + 1) * D] for c in range(kappa)] for me in ins])
        if R.take(kappa * D) != [v for col in c_parent for v in col]:
            raise VerifyError(f"{lane.decode()} lane: RLC commitment mismatch")
        X_parent = mix([[[me["X"][rho * m_in + j] for rho in range(D)] for j in range(m_in)] for me in ins])
        rows = t + nb
        y_re = mix([[[me["y"][row][rho][0] for rho in range(D)] for row in range(rows)] for me in ins])
        y_im = mix([[[me["y"][row][rho][1] for rho in range(D)] for row in range(rows)] for me in ins])
        # DEC: children X are the balanced base-b digits of X_parent
        Xp = np.array([[centered(X_parent[j][rho]) for j in range(m_in)] for rho in range(D)], np.int64)
        if np.abs(Xp).max(initial=0) >= (1 << 31):
            raise VerifyError("DEC: X out of range")
        planes, _ = split_b(Xp.astype(np.int32), self.k_rho, self.b)
        children = []
        csum = [0] * (kappa * D)
        ysum_re = [[0] * D for _ in range(rows)]
        ysum_im = [[0] * D for _ in range(rows)]
        for ci in range(self.k_rho):
            c = R.take(kappa * D)
            ycore = [R.ks(D) for _ in range(t)]
            ybus = [R.ks(D) for _ in range(nb)]
            yrows = ycore + ybus
            Xc = [int(v) % Q for v in planes[ci].astype(np.int64).reshape(-1)]
            children.append(self._me(c, Xc, r, yrows, digest))
            pw = pow(self.b, ci, Q)
            csum = [(a + pw * v) % Q for a, v in zip(csum, c)]
            for row in range(rows):
                for rho in range(D):
                    ysum_re[row][rho] = (ysum_re[row][rho] + pw * yrows[row][rho][0]) % Q
                    ysum_im[row][rho] = (ysum_im[row][rho] + pw * yrows[row][rho][1]) % Q
        # verify_dec_public: sum_i b^i (c, y) of the children = the parent's
        if csum != [v for col in c_parent for v in col]:
            raise VerifyError(f"{lane.decode()} lane: DEC commitment check failed")
        if ysum_re != y_re or ysum_im != y_im:
            raise VerifyError(f"{lane.decode()} lane: DEC y check failed")
        if rec is not None:
            parent_rows = [[(a, b) for a, b in zip(y_re[row], y_im[row])] for row in range(rows)]
            rec.update(rhos=[list(v) for v in rhos], children=children,
                       parent=self._me([v for col in c_parent for v in col],
                                       [X_parent[j][rho] for rho in range(D) for j in range(m_in)], r, parent_rows,
                                       digest))
        return children

    def verify_step_struct(self, x, S):
        """Check one step's proof in StepProof struct order (neo_gpu_shard_step_proof):
        its proof-carried fields go through verify_step, and every field the
        replay derives (ME claims' r, X, digests, the RLC parent, the public
        challenges) must equal the struct's, word for word."""
        from .step_proof import read_step, to_transcript_order, write_step
        try:
            f = read_step(S)
            P, _ = to_transcript_order(f, self.t, self.bus.bus_cols, self.ell_n)
        except (ValueError, IndexError, KeyError, TypeError) as e:
            raise VerifyError(f"malformed struct-order proof: {e}")
        rec = {}
        self.verify_step(x, P, record=rec, _struct=True)
        if not np.array_equal(write_step(rec, self.kappa, 1 << self.ell_d), np.asarray(S, np.uint64)):
            raise VerifyError("struct-order fields differ from the verifier's replay")
        return True

    # ---------------------------------------------------------------- memory --
    def set_twist_init(self, i, init):
        """The public MemInit of Twist instance i for the following steps."""
        init = [(int(a), int(v) % Q) for a, v in init]
        if any(b[0] <= a[0] for a, b in zip(init, init[1:])):
            raise VerifyError("MemInit::Sparse must be strictly increasing by address")
        self.twist[i] = dict(self.twist[i], init=init)
        fs = []
        for a, v in init:
            fs += [a, v]
        self.twist_digest[i] = digest_fields(b"twist/init/sparse" if init else b"twist/init/zero", fs)

    @staticmethod
    def _init_at(init, r_addr):
        """eval_init_at_r_addr (neo-memory/src/mem_init.rs:133-170)."""
        acc = ZERO
        for a, v in init:
            chi = ONE
            for bit, r in enumerate(r_addr):
                chi = kmulp(chi, r if (a >> bit) & 1 else ksub(ONE, r))
            acc = kadd(acc, kmulp((int(v) % Q, 0), chi))
        return acc

    @staticmethod
    def _eq_bits(bits, u):
        """eq_bits_prod with eq_bit_affine(b, u) = b (2u - 1) + (1 - u) (neo-memory/src/bit_ops.rs:6-20)."""
        acc = ONE
        for b, x in zip(bits, u):
            acc = kmulp(acc, kadd(kmulp(b, ksub(kadd(x, x), ONE)), ksub(ONE, x)))
        return acc

    def _bitness_weights(self, r0, n, sep):
        """bitness_weights (memory_sidecar/utils.rs:43-71): powers of r_cycle[0] + sep."""
        base = ((r0[0] + sep) % Q, r0[1])
        if base in (ZERO, ONE, (Q - 1, 0)):
            base = ((base[0] + 1) % Q, base[1])
        if base == ZERO:
            base = ONE
        out, cur = [], ONE
        for _ in range(n):
            out.append(cur)
            cur = kmulp(cur, base)
        return out

    def _bitness_expected(self, chi, r0, opens, sep):
        acc = ZERO
        for w, b in zip(self._bitness_weights(r0, len(opens), sep), opens):
            acc = kadd(acc, kmulp(w, kmulp(b, ksub(b, ONE))))
        return kmulp(chi, acc)

    @staticmethod
    def _lt_eval(jp, j):
        """lt_eval (neo-memory/src/mle.rs:7-24)."""
        ell = len(j)
        suffix = [ONE] * (ell + 1)
        for i in range(ell - 1, -1, -1):
            e = kadd(kmulp(ksub(ONE, jp[i]), ksub(ONE, j[i])), kmulp(jp[i], j[i]))
            suffix[i] = kmulp(suffix[i + 1], e)
        acc = ZERO
        for i in range(ell):
            acc = kadd(acc, kmulp(kmulp(ksub(ONE, jp[i]), j[i]), suffix[i + 1]))
        return acc

    def _bind_claim_sums(self, prefix, sums, labels):
        """bind_batched_claim_sums (memory_sidecar/transcript.rs:12-26)."""
        self.tr.append_message(prefix, le64(len(sums)))
        for i, (sm, lab) in enumerate(zip(sums, labels)):
            self.tr.append_message(b"addr_batch/label", lab)
            self.tr.append_message(b"addr_batch/idx", le64(i))
            self._k(b"addr_batch/claimed_sum", sm)

    def _time_claim_plan(self):
        """RouteATimeClaimPlan (memory_sidecar/claim_plan.rs:42-187): (label, degree, dynamic)."""
        plan = [(b"ccs/time", self.d_sc, True)]
        for s in self.shout:
            plan += [(b"shout/value", 3, True), (b"shout/adapter", 2 + s["ell_addr"], True), (b"shout/bitness", 3, False)]
        for w in self.twist:
            plan += [(b"twist/read_check", 3 + w["ell_addr"], True), (b"twist/write_check", 3 + w["ell_addr"], True),
                     (b"twist/bitness", 3, False)]
        return plan

    # -------------------------------------------------------------- fold step --
    def verify_step(self, x, P, record=None, _struct=False):
        """Check one step's proof words against the public input x = z[:m_in]
        (and the step's public memory instances); on success the verified DEC
        children become the accumulator and the val-lane children are added to
        val_obligations.  record (a dict) receives the step's fields in the
        struct order of StepProof (oracle/step_proof.py).  _struct: P was rebuilt
        from a struct-order proof, which carries neither the words the verifier
        derives itself (Twist address finals, r_val) nor a one-instance lane's
        sampled rho."""
        rec = record if record is not None else {}
        self._struct = _struct
        tr, t, ell_n, ell_d, d_sc = self.tr, self.t, self.ell_n, self.ell_d, self.d_sc
        idx, kappa, m_in = self.step_idx, self.kappa, self.m_in
        bus, nb = self.bus, self.bus.bus_cols
        R = Reader(P)
        n_acc = len(self.acc)
        k = 1 + n_acc
        xv = [int(v) % Q for v in np.asarray(x, np.uint64).reshape(-1)][:m_in]
        c_mcs = R.take(kappa * D)
        Xm = [int(v) % Q for v in decomp_b2(np.array(xv, np.uint64)).astype(np.int64).reshape(-1)]
        # absorb_step_memory (memory_sidecar/memory.rs:86-124)
        tr.append_message(b"step/absorb_memory_start")
        tr.append_message(b"step/lut_count", le64(len(self.shout)))
        for i, sd in enumerate(self.shout):
            tr.append_message(b"step/lut_idx", le64(i))
            tr.append_message(b"shout/k", le64(sd["k"]))
            tr.append_message(b"shout/d", le64(sd["d"]))
            tr.append_message(b"shout/n_side", le64(sd["n_side"]))
            tr.append_message(b"shout/steps", le64(bus.chunk))
            tr.append_message(b"shout/ell", le64(sd["ell"]))
            tr.append_message(b"shout/table_digest", self.shout_digest[i])
        tr.append_message(b"step/mem_count", le64(len(self.twist)))
        for i, w in enumerate(self.twist):
            tr.append_message(b"step/mem_idx", le64(i))
            tr.append_message(b"twist/k", le64(w["k"]))
            tr.append_message(b"twist/d", le64(w["d"]))
            tr.append_message(b"twist/n_side", le64(w["n_side"]))
            tr.append_message(b"twist/steps", le64(bus.chunk))
            tr.append_message(b"twist/ell", le64(w["ell"]))
            tr.append_message(b"twist/init_digest", self.twist_digest[i])
        tr.append_message(b"step/absorb_memory_done")
        # bind_header_and_instances_with_digest (engines/utils.rs:83-137)
        tr.append_message(b"phase/pi-ccs")
        tr.append_message(b"neo/ccs/header/v1")
        tr.append_u64s(b"ccs/header", [64, 2, self.lam, ell_n + ell_d, d_sc, abs(self.slack)])
        tr.append_message(b"ccs/slack_sign", bytes([1 if self.slack >= 0 else 0]))
        tr.append_message(b"neo/ccs/instances")
        tr.append_u64s(b"dims", [self.n, self.m, t])
        for dgt in self.digest:
            tr.append_fields(b"mat_digest", [int(dgt)])
        tr.append_message(b"neo/ccs/poly")
        tr.append_u64s(b"arity", [t])
        tr.append_u64s(b"terms_len", [len(self.ccs.f_terms)])
        for coeff, exps in sorted(self.ccs.f_terms, key=lambda te: te[1]):
            tr.append_fields(b"coeff", [coeff % Q])
            tr.append_u64s(b"exps", exps)
        tr.append_fields(b"x", xv)
        tr.append_u64s(b"m_in", [m_in])
        tr.append_fields(b"c_data", c_mcs)
        # bind_me_inputs (engines/utils.rs:139-181)
        tr.append_message(b"neo/ccs/me_inputs/v2")
        tr.append_u64s(b"me_count", [n_acc])
        for me in self.acc:
            tr.append_fields(b"c_data_in", me["c"])
            tr.append_u64s(b"m_in_in", [me["m_in"]])
            tr.append_fields(b"r_in", [v for rk in me["r"] for v in rk])
            tr.append_fields(b"y_elem", [v for row in me["y"] for e in row for v in e])
        # sample_challenges (engines/utils.rs:184-212)
        tr.append_message(b"neo/ccs/chals/v1")
        ck = lambda: tuple(int(v) for v in tr.challenge_fields(b"chal/k", 2))
        alpha = [ck() for _ in range(ell_d)]
        beta = [ck() for _ in range(ell_d + ell_n)]
        gamma = ck()
        beta_a, beta_r = beta[:ell_d], beta[ell_d:]
        T = self._initial_sum(alpha, gamma, k)
        rec.update(alpha=alpha, beta_a=beta_a, beta_r=beta_r, gamma=gamma, T=T, shout=None, twist=[], val_eval=None,
                   val=None, cpu_me_val=[])
        if R.k() != T:
            raise VerifyError("initial sum mismatch: proof claims a different value than the public T")
        self._k(b"sumcheck/initial_sum", T)
        r_cycle = self._sample_ext_point(b"route_a/r_cycle", b"route_a/cycle/0", b"route_a/cycle/1", ell_n)

        # ---- verify_shout_addr_pre_time (memory.rs:623-816) ----
        shout_pre = []
        r_addr_s = []
        if self.shout:
            ea = self.shout[0]["ell_addr"]
            if any(sd["ell_addr"] != ea for sd in self.shout):
                raise VerifyError("Shout: batched addr-pre requires uniform ell_addr")
            sums = R.ks(len(self.shout))
            active = R.take(1)[0]
            if active >> len(self.shout):
                raise VerifyError("shout_addr_pre active_mask has bits set out of range")
            tr.append_message(b"shout/addr_pre_time/step_idx", le64(idx))
            self._bind_claim_sums(b"shout/addr_pre_time/claimed_sums", sums, [b"shout/addr_pre"] * len(sums))
            act = [i for i in range(len(self.shout)) if (active >> i) & 1]
            if not act:
                tr.append_message(b"shout/addr_pre_time/no_sumcheck", le64(idx))
                r_addr_s = self._sample_ext_point(b"shout/addr_pre_time/no_sumcheck/r_addr",
                                                  b"shout/addr_pre_time/no_sumcheck/r_addr/0",
                                                  b"shout/addr_pre_time/no_sumcheck/r_addr/1", ea)
                finals = []
            else:
                r_addr_s, finals = self._batched_ds(b"shout/addr_pre_time", idx, [b"shout/addr_pre"] * len(act),
                                                    [2] * len(act), [sums[i] for i in act], ea, R)
            rec["shout"] = dict(sums=sums, active=active, polys=self.last_polys if act else [], r_addr=r_addr_s)
            if R.ks(ea) != r_addr_s:
                raise VerifyError("shout_addr_pre r_addr mismatch: transcript-derived vs proof")
            pos = 0
            for i, sd in enumerate(self.shout):
                is_active = i in act
                fin = finals[pos] if is_active else ZERO
                pos += 1 if is_active else 0
                tab_eval = ZERO
                if is_active:
                    chi = chi_table(r_addr_s)
                    for a, v in enumerate(list(sd["table"])[:1 << ea]):
                        tab_eval = kadd(tab_eval, kmulp((int(v) % Q, 0), chi[a]))
                shout_pre.append(dict(active=is_active, claim=sums[i], final=fin, table_eval=tab_eval))

        # ---- verify_twist_addr_pre_time (memory.rs:818-903) ----
        twist_pre = []
        for i, w in enumerate(self.twist):
            ea = w["ell_addr"]
            labels = [b"twist/read_addr_pre", b"twist/write_addr_pre"]
            tr.append_message(b"twist/addr_pre_time/claim_idx", le64(i))
            self._bind_claim_sums(b"twist/addr_pre_time/claimed_sums", [ZERO, ZERO], labels)
            r_addr, finals = self._batched_ds(b"twist/addr_pre_time", i, labels, [2, 2], [ZERO, ZERO], ea, R)
            rec["twist"].append(dict(polys=self.last_polys, r_addr=r_addr, finals=finals))
            if R.ks(ea) != r_addr:
                raise VerifyError("twist addr_pre r_addr mismatch: transcript-derived vs proof")
            if not _struct and R.ks(2) != finals:
                raise VerifyError("twist addr_pre finals mismatch")
            twist_pre.append(dict(r_addr=r_addr, read=finals[0], write=finals[1]))

        # ---- verify_route_a_batched_time (route_a_time.rs:159-290) ----
        plan = self._time_claim_plan()
        labels = [p_[0] for p_ in plan]
        degs = [p_[1] for p_ in plan]
        # claimed sums: the CCS claim is the public T, static claims are 0, the
        # dynamic memory claims are those of the proof's first round, p(0) + p(1)
        first = Reader(R.P[R.i:R.i + sum(2 * (d + 1) for d in degs)])
        sums = []
        for (lab, deg, dyn) in plan:
            co = first.ks(deg + 1)
            p1 = ZERO
            for c in co:
                p1 = kadd(p1, c)
            sums.append(kadd(co[0], p1) if dyn else ZERO)
        sums[0] = T
        tr.append_message(b"batched/dynamic_bind/len", le64(len(plan)))
        for ci, (lab, deg, dyn) in enumerate(plan):
            tr.append_message(b"batched/dynamic_bind/claim_label", lab)
            tr.append_message(b"batched/dynamic_bind/claim_idx", le64(ci))
            tr.append_message(b"batched/dynamic_bind/degree_bound", le64(deg))
            tr.append_message(b"batched/dynamic_bind/is_dynamic", bytes([1 if dyn else 0]))
            if dyn:
                self._k(b"batched/dynamic_bind/claimed_sum", sums[ci])
        r_time, finals = self._batched_ds(b"shard/batched_time", idx, labels, degs, sums, ell_n, R)
        rec["time"] = dict(sums=list(sums), degs=list(degs), labels=list(labels), polys=self.last_polys)
        rec["r_time"] = r_time
        # ---- CCS Ajtai rounds (verify_sumcheck_rounds_ds with domain ccs/ajtai) ----
        running = finals[0]
        tr.append_message(b"sc/domain", b"ccs/ajtai")
        tr.append_message(b"sc/inst_idx", le64(idx))
        self._k(b"sc/claimed_sum", running)
        alpha_p = []
        rec["ajtai_polys"] = []
        for rd in range(ell_d):
            co = R.ks(d_sc + 1)
            rec["ajtai_polys"].append(co)
            p1 = ZERO
            for c in co:
                p1 = kadd(p1, c)
            if kadd(co[0], p1) != running:
                raise VerifyError(f"Pi_CCS Ajtai round {rd}: p(0) + p(1) != running claim")
            for c in co:
                self._k(b"sumcheck/round/coeff", c)
            r = self._chal(b"sumcheck/challenge/0", b"sumcheck/challenge/1")
            alpha_p.append(r)
            running = kpoly(co, r)
        tr.append_message(b"sc/domain_end", b"ccs/ajtai")
        tr.append_message(b"sc/inst_idx_end", le64(idx))
        if R.k() != running:
            raise VerifyError("Pi_CCS sumcheck_final mismatch")
        rec["alpha_p"], rec["final"] = alpha_p, running
        fold_digest = tr.digest32()
        # ---- ME outputs (core rows + bus openings) and the Pi_CCS terminal identity ----
        y_out = [[R.ks(D) for _ in range(t)] for _ in range(k)]
        ysc_out = [R.ks(t) for _ in range(k)]
        bus_y = []
        for i in range(k):
            rows = [R.ks(D) for _ in range(nb)]
            bsc = R.ks(nb)
            if self._yscalars(rows) != bsc:
                raise VerifyError(f"ME output {i}: bus y_scalars do not recompose the bus y rows")
            bus_y.append((rows, bsc))
        for i in range(k):
            if self._yscalars(y_out[i]) != ysc_out[i]:
                raise VerifyError(f"Pi_CCS output {i}: y_scalars do not recompose y")
        r_in = self.acc[0]["r"] if n_acc else None
        rhs = self._terminal_rhs(alpha, beta_a, beta_r, gamma, r_time, alpha_p, y_out, r_in)
        if rhs != running:
            raise VerifyError("Pi_CCS terminal identity check failed")
        srcs = [dict(c=c_mcs, X=Xm)] + [dict(c=me["c"], X=me["X"]) for me in self.acc]
        outs = [self._me(s_["c"], s_["X"], r_time, y_out[i] + bus_y[i][0], fold_digest) for i, s_ in enumerate(srcs)]
        rec["ccs_out"] = outs

        # ---- Twist val-eval batch (memory.rs:2088-2170) ----
        has_prev = self.prev is not None
        val_claims, r_val, vfin, vsums = [], [], [], []
        if self.twist:
            vplan = []
            for i, w in enumerate(self.twist):
                ea = w["ell_addr"]
                vplan += [(b"twist/val_eval_lt", ea + 3, 0), (b"twist/val_eval_total", ea + 2, 1)]
                if has_prev:
                    vplan.append((b"twist/rollover_prev_total", ea + 2, 2))
            vsums = R.ks(len(vplan))
            tr.append_message(b"twist/val_eval/batch_start", le64(len(self.twist)))
            tr.append_message(b"twist/val_eval/step_idx", le64(idx))
            tr.append_message(b"twist/val_eval/claimed_sums_len", le64(len(vplan)))
            for ci, ((lab, deg, tag), sm) in enumerate(zip(vplan, vsums)):
                tr.append_message(b"twist/val_eval/claim_idx", le64(ci))
                tr.append_message(b"twist/val_eval/claim_kind", bytes([tag]))
                self._k(b"twist/val_eval/claimed_sum", sm)
            r_val, vfin = self._batched_ds(b"twist/val_eval_batch", idx, [v[0] for v in vplan], [v[1] for v in vplan],
                                           vsums, ell_n, R)
            rec["val_eval"] = dict(sums=vsums, polys=self.last_polys, r_val=r_val, has_prev=has_prev)
            tr.append_message(b"twist/val_eval/batch_done")
            if not _struct and R.ks(ell_n) != r_val:
                raise VerifyError("twist val-eval r_val mismatch")
            # CPU ME claims at r_val (ts_common.rs:100-258): the current and previous MCS
            fork = tr.clone_state()
            fork.append_message(b"fork", b"cpu_bus/me_digest_val")
            vdigest = fork.digest32()
            vsrcs = [(c_mcs, Xm)] + ([(self.prev["c"], self.prev["X"])] if has_prev else [])
            for c_, X_ in vsrcs:
                rows = [R.ks(D) for _ in range(t + nb)]
                ysc = R.ks(t + nb)
                if self._yscalars(rows) != ysc:
                    raise VerifyError("CPU ME(val): y_scalars do not recompose y")
                val_claims.append(self._me(c_, X_, r_val, rows, vdigest))
            rec["cpu_me_val"] = val_claims

        # ---- verify_route_a_memory_step (memory.rs:1671-2380) ----
        if self.shout or self.twist:
            chi_c = keq(r_time, r_cycle)
            o0 = bus_y[0][1]  # bus y_scalars of the MCS output at r_time
            ci = 1
            for i, (sd, sc) in enumerate(zip(self.shout, bus.shout)):
                ea = sd["ell_addr"]
                bits = [o0[c] for c in sc["addr_bits"]]
                has, val = o0[sc["has_lookup"]], o0[sc["val"]]
                pre = shout_pre[i]
                if self._bitness_expected(chi_c, r_cycle[0], bits + [has], 0x5348_4F55_54 + i) != finals[ci + 2]:
                    raise VerifyError("shout/bitness terminal value mismatch")
                if kmulp(chi_c, kmulp(has, val)) != finals[ci]:
                    raise VerifyError("shout value terminal value mismatch")
                if kmulp(chi_c, kmulp(has, self._eq_bits(bits, r_addr_s))) != finals[ci + 1]:
                    raise VerifyError("shout adapter terminal value mismatch")
                if sums[ci] != pre["claim"]:
                    raise VerifyError("shout value claimed sum != addr claimed sum")
                if pre["active"]:
                    if kmulp(pre["table_eval"], sums[ci + 1]) != pre["final"]:
                        raise VerifyError("shout addr terminal value mismatch")
                elif pre["claim"] != ZERO or sums[ci + 1] != ZERO or pre["final"] != ZERO:
                    raise VerifyError("shout addr-pre skipped but a claim is nonzero")
                ci += 3
            lt = self._lt_eval(r_val, r_time) if self.twist else ZERO
            per = 3 if has_prev else 2
            for i, (w, tc) in enumerate(zip(self.twist, bus.twist)):
                pre = twist_pre[i]
                r_addr = pre["r_addr"]
                ra = [o0[c] for c in tc["ra_bits"]]
                wa = [o0[c] for c in tc["wa_bits"]]
                hr, hw, wv, rv, inc = (o0[tc[n]] for n in ("has_read", "has_write", "wv", "rv", "inc"))
                if sums[ci] != pre["read"] or sums[ci + 1] != pre["write"]:
                    raise VerifyError("twist read/write check claimed sum != addr-pre final")
                if self._bitness_expected(chi_c, r_cycle[0], ra + wa + [hr, hw], 0x5457_4953_54 + i) != finals[ci + 2]:
                    raise VerifyError("twist/bitness terminal value mismatch")
                claimed_val = kadd(self._init_at(w.get("init", []), r_addr), vsums[per * i])
                exp_r = kmulp(chi_c, kmulp(hr, kmulp(ksub(claimed_val, rv), self._eq_bits(ra, r_addr))))
                if exp_r != finals[ci]:
                    raise VerifyError("twist/read_check terminal value mismatch")
                exp_w = kmulp(chi_c, kmulp(hw, kmulp(ksub(ksub(wv, claimed_val), inc), self._eq_bits(wa, r_addr))))
                if exp_w != finals[ci + 1]:
                    raise VerifyError("twist/write_check terminal value mismatch")
                # val-eval terminals against the CPU ME openings at r_val
                ov = val_claims[0]["ysc"][t:]
                inc_v = kmulp(ov[tc["has_write"]], kmulp(ov[tc["inc"]], self._eq_bits([ov[c] for c in tc["wa_bits"]],
                                                                                     r_addr)))
                if kmulp(inc_v, lt) != vfin[per * i]:
                    raise VerifyError("twist/val_eval_lt terminal value mismatch")
                if inc_v != vfin[per * i + 1]:
                    raise VerifyError("twist/val_eval_total terminal value mismatch")
                if has_prev:
                    op = val_claims[1]["ysc"][t:]
                    inc_p = kmulp(op[tc["has_write"]], kmulp(op[tc["inc"]],
                                                             self._eq_bits([op[c] for c in tc["wa_bits"]], r_addr)))
                    if inc_p != vfin[per * i + 2]:
                        raise VerifyError("twist/rollover_prev_total terminal value mismatch")
                    # Init_i(r_addr) == Init_{i-1}(r_addr) + PrevTotal(i)
                    prev_init = self._init_at(self.prev["init"][i], r_addr)
                    if self._init_at(w.get("init", []), r_addr) != kadd(prev_init, vsums[per * i + 2]):
                        raise VerifyError("twist rollover init check failed")
                ci += 3

        # ---- main lane, val lane ----
        rec["main"] = {}
        children = self._lane(b"main", idx, outs, r_time, fold_digest, R, rec["main"])
        if val_claims:
            tr.append_message(b"fold/val_lane_start", le64(idx))
            rec["val"] = {}
            self.val_obligations += self._lane(b"val", idx, val_claims, r_val, vdigest, R, rec["val"])
        tr.append_message(b"fold/step_done", le64(idx))
        R.done()
        self.acc = children
        if self.twist:
            self.prev = dict(c=c_mcs, X=Xm, init=[list(w.get("init", [])) for w in self.twist])
        self.step_idx += 1
        return True
