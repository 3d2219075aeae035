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
        self.shout, self.twist = self.mem.get("shout", []), self.mem.get("twist", [])
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
        if self.shout or self.twist:
            raise NotImplementedError("memory sidecar verification")

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
        for rd in range(n_rounds):
            tr.append_message(b"batched/round_idx", le64(rd))
            polys = [R.ks(deg + 1) for deg in degs]
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
    def _lane(self, lane, idx, ins, r, digest, R):
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
        if [centered(v) for v in R.take(k * D)] != [int(v) for v in rhos.reshape(-1)]:
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
        return children

    # -------------------------------------------------------------- fold step --
    def verify_step(self, x, P):
        """Check one step's proof words against the public input x = z[:m_in];
        on success the verified DEC children become the accumulator."""
        tr, t, ell_n, ell_d, d_sc = self.tr, self.t, self.ell_n, self.ell_d, self.d_sc
        idx, kappa, m_in = self.step_idx, self.kappa, self.m_in
        R = Reader(P)
        n_acc = len(self.acc)
        k = 1 + n_acc
        d_pad = 1 << ell_d
        xv = [int(v) % Q for v in np.asarray(x, np.uint64).reshape(-1)][:m_in]
        c_mcs = R.take(kappa * D)
        Xm = [int(v) % Q for v in decomp_b2(np.array(xv, np.uint64)).astype(np.int64).reshape(-1)]
        # absorb_step_memory (memory_sidecar/memory.rs:86-124), no instances
        tr.append_message(b"step/absorb_memory_start")
        tr.append_message(b"step/lut_count", le64(0))
        tr.append_message(b"step/mem_count", le64(0))
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
        if R.k() != T:
            raise VerifyError("initial sum mismatch: proof claims a different value than the public T")
        self._k(b"sumcheck/initial_sum", T)
        self._sample_ext_point(b"route_a/r_cycle", b"route_a/cycle/0", b"route_a/cycle/1", ell_n)
        # bind_batched_dynamic_claims (memory_sidecar/transcript.rs:37-63): the CCS claim alone
        labels, degs, sums = [b"ccs/time"], [d_sc], [T]
        tr.append_message(b"batched/dynamic_bind/len", le64(1))
        tr.append_message(b"batched/dynamic_bind/claim_label", b"ccs/time")
        tr.append_message(b"batched/dynamic_bind/claim_idx", le64(0))
        tr.append_message(b"batched/dynamic_bind/degree_bound", le64(d_sc))
        tr.append_message(b"batched/dynamic_bind/is_dynamic", bytes([1]))
        self._k(b"batched/dynamic_bind/claimed_sum", T)
        r_time, finals = self._batched_ds(b"shard/batched_time", idx, labels, degs, sums, ell_n, R)
        # CCS Ajtai rounds (verify_sumcheck_rounds_ds with domain ccs/ajtai)
        running = finals[0]
        tr.append_message(b"sc/domain", b"ccs/ajtai")
        tr.append_message(b"sc/inst_idx", le64(idx))
        self._k(b"sc/claimed_sum", running)
        alpha_p = []
        for rd in range(ell_d):
            co = R.ks(d_sc + 1)
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
        fold_digest = tr.digest32()
        # ME outputs (core rows) and the terminal identity
        y_out = [[R.ks(D) for _ in range(t)] for _ in range(k)]
        ysc_out = [R.ks(t) for _ in range(k)]
        for i in range(k):
            if self._yscalars(y_out[i]) != ysc_out[i]:
                raise VerifyError(f"Pi_CCS output {i}: y_scalars do not recompose y")
        r_in = self.acc[0]["r"] if n_acc else None
        rhs = self._terminal_rhs(alpha, beta_a, beta_r, gamma, r_time, alpha_p, y_out, r_in)
        if rhs != running:
            raise VerifyError("Pi_CCS terminal identity check failed")
        srcs = [dict(c=c_mcs, X=Xm)] + [dict(c=me["c"], X=me["X"]) for me in self.acc]
        outs = [self._me(s["c"], s["X"], r_time, y_out[i], fold_digest) for i, s in enumerate(srcs)]
        children = self._lane(b"main", idx, outs, r_time, fold_digest, R)
        tr.append_message(b"fold/step_done", le64(idx))
        R.done()
        self.acc = children
        self.step_idx += 1
        return True
