"""CPU restatement of one Neo fold step (main lane, no Twist/Shout).

TEST INFRASTRUCTURE ONLY: the parity checker for neo_gpu_shard_fold_step and
the CPU-baseline leg of bench.py.  It composes the oracle's C primitives in
the order of fold_shard_prove_impl (crates/neo-fold/src/shard.rs:1803-2180)
and prove_rlc_dec_lane (shard.rs:1170-1331), with the transcript calls of
engines/utils.rs:83-212, memory_sidecar/route_a_time.rs:28-152,
memory_sidecar/sumcheck_ds.rs:11-77 and sumcheck.rs:124-456, and emits the
same canonical step-proof word dump as the CUDA library.
"""
import struct

import numpy as np

from . import (CcsOracle, Transcript, ccs_digest, commit_digits, decomp_b2, interpolate, k_mul, poly_eval_k,
               rlc_mix, split_b, lib, u64)

Q = (1 << 64) - (1 << 32) + 1
D = 54


def le64(v):
    return struct.pack("<Q", v)


def kadd(a, b):
    return ((a[0] + b[0]) % Q, (a[1] + b[1]) % Q)


def kmulp(a, b):
    return ((a[0] * b[0] + 7 * a[1] * b[1]) % Q, (a[0] * b[1] + a[1] * b[0]) % Q)


def header_params(ell, d_sc):
    """goldilocks_auto_r1cs_ccs + extension_check (crates/neo-params/src/lib.rs:181-304)."""
    q2 = Q * Q
    for lam in range(127, 95, -1):
        rhs = (1 << lam) * ell * d_sc
        if q2 < rhs:
            continue
        slack = q2.bit_length() - rhs.bit_length()
        if q2 < (rhs << slack):
            slack -= 1
        if slack >= 2:
            return lam, slack
    raise ValueError("no lambda")


def rot_int(a):
    """integer rot(a): column t = a X^t mod Phi_81"""
    R = np.zeros((D, D), np.int64)
    col = np.array(a, np.int64)
    for t in range(D):
        R[:, t] = col
        last = col[-1]
        nxt = np.zeros(D, np.int64)
        nxt[1:] = col[:-1]
        nxt[0] -= last
        nxt[27] -= last
        col = nxt
    return R


class OracleShard:
    def __init__(self, ccs, pp, m_in=1, k_rho=12, app_label=b"neo/shard", threads=0):
        self.ccs, self.pp = ccs, np.ascontiguousarray(pp, np.uint64)
        self.kappa = pp.shape[0]
        self.m_in, self.k_rho, self.b = m_in, k_rho, 2
        self.n, self.m, self.t = ccs.n, ccs.m, ccs.t
        self.ell_n = (self.n - 1).bit_length()
        self.ell_d = 6
        self.d_sc = max(ccs.f_degree + 1, 2 * self.b + 2)
        self.lam, self.slack = header_params(self.ell_n + self.ell_d, self.d_sc)
        self.digest = ccs_digest(ccs)
        self.tr = Transcript(app_label)
        self.acc = []        # ME instances
        self.acc_Z = []      # digit matrices [54][m]
        self.step_idx = 0
        self.threads = threads

    def _k(self, label, v):
        self.tr.append_fields(label, np.array(v, np.uint64))

    def fold_step(self, z):
        tr, t, ell_n, ell_d, d_sc = self.tr, self.t, self.ell_n, self.ell_d, self.d_sc
        idx, kappa, m_in = self.step_idx, self.kappa, self.m_in
        n_acc = len(self.acc)
        k = 1 + n_acc
        d_pad = 1 << ell_d
        P = []
        Zm = decomp_b2(z)
        c_mcs = commit_digits(self.pp, Zm, self.threads).reshape(-1)
        P += [int(v) for v in c_mcs]
        x = [int(v) % Q for v in np.asarray(z[:m_in], np.uint64)]
        Xm = [int(v) % Q for v in Zm[:, :m_in].astype(np.int64).reshape(-1)]
        mcs = dict(c=c_mcs, X=Xm, m_in=m_in)
        # bind_header_and_instances_with_digest
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
        tr.append_fields(b"x", x)
        tr.append_u64s(b"m_in", [m_in])
        tr.append_fields(b"c_data", c_mcs)
        # bind_me_inputs
        tr.append_message(b"neo/ccs/me_inputs/v2")
        tr.append_u64s(b"me_count", [n_acc])
        for me in self.acc:
            tr.append_fields(b"c_data_in", me["c"])
            tr.append_u64s(b"m_in_in", [me["m_in"]])
            tr.append_fields(b"r_in", np.asarray(me["r"], np.uint64).reshape(-1))
            tr.append_fields(b"y_elem", np.asarray(me["y"], np.uint64).reshape(-1))
        # sample_challenges
        tr.append_message(b"neo/ccs/chals/v1")
        ck = lambda: tuple(int(v) for v in tr.challenge_fields(b"chal/k", 2))
        alpha = [ck() for _ in range(ell_d)]
        beta = [ck() for _ in range(ell_d + ell_n)]
        gamma = ck()
        beta_a, beta_r = beta[:ell_d], beta[ell_d:]
        # claimed_initial_sum_from_inputs
        T = (0, 0)
        if k >= 2:
            chi_a = []
            for rho in range(d_pad):
                w = (1, 0)
                for bit in range(ell_d):
                    a = alpha[bit]
                    w = kmulp(w, a if (rho >> bit) & 1 else ((1 - a[0]) % Q, (-a[1]) % Q))
                chi_a.append(w)
            gk = (1, 0)
            for _ in range(k):
                gk = kmulp(gk, gamma)
            inner, gkj = (0, 0), (1, 0)
            for j in range(t):
                gi = (1, 0)
                for me in self.acc:
                    gi = kmulp(gi, gamma)
                    ye = (0, 0)
                    for rho in range(d_pad):
                        yv = me["y"][j][rho]
                        ye = kadd(ye, kmulp((int(yv[0]), int(yv[1])), chi_a[rho]))
                    inner = kadd(inner, kmulp(kmulp(gi, gkj), ye))
                gkj = kmulp(gkj, gk)
            T = kmulp(gk, inner)
        self._k(b"sumcheck/initial_sum", T)
        P += list(T)
        for i in range(ell_n):
            tr.append_message(b"route_a/r_cycle", le64(i))
            tr.challenge_field(b"route_a/cycle/0")
            tr.challenge_field(b"route_a/cycle/1")
        # oracle
        Zall = np.stack([Zm] + self.acc_Z)
        rin = np.array(self.acc[0]["r"], np.uint64) if n_acc else None
        orc = CcsOracle(self.ccs, Zall, 2, np.array(alpha, np.uint64), np.array(beta_a, np.uint64),
                        np.array(beta_r, np.uint64), np.array(gamma, np.uint64), rin, ell_d, ell_n, d_sc)
        xs = np.array([[i, 0] for i in range(d_sc + 1)], np.uint64)
        tr.append_message(b"batched/dynamic_bind/len", le64(1))
        tr.append_message(b"batched/dynamic_bind/claim_label", b"ccs/time")
        tr.append_message(b"batched/dynamic_bind/claim_idx", le64(0))
        tr.append_message(b"batched/dynamic_bind/degree_bound", le64(d_sc))
        tr.append_message(b"batched/dynamic_bind/is_dynamic", bytes([1]))
        self._k(b"batched/dynamic_bind/claimed_sum", T)
        tr.append_message(b"sc/domain", b"shard/batched_time")
        tr.append_message(b"sc/inst_idx", le64(idx))
        running = np.array(T, np.uint64)
        r_time = []
        for rd in range(ell_n):
            tr.append_message(b"batched/round_idx", le64(rd))
            ys = orc.evals_at(xs)
            s01 = kadd((int(ys[0, 0]), int(ys[0, 1])), (int(ys[1, 0]), int(ys[1, 1])))
            if s01 != (int(running[0]), int(running[1])):
                raise AssertionError(f"batched round {rd}: invariant")
            co = interpolate(xs, ys)
            tr.append_message(b"batched/claim_label", b"ccs/time")
            tr.append_message(b"batched/claim_idx", le64(0))
            for c in co:
                self._k(b"batched/round/coeff", c)
            r = np.array([tr.challenge_field(b"batched/challenge/0"), tr.challenge_field(b"batched/challenge/1")],
                         np.uint64)
            r_time.append(r)
            running = poly_eval_k(co, r)
            orc.fold(r)
            P += [int(v) for v in co.reshape(-1)]
        tr.append_message(b"sc/domain_end", b"shard/batched_time")
        tr.append_message(b"sc/inst_idx_end", le64(idx))
        tr.append_message(b"sc/domain", b"ccs/ajtai")
        tr.append_message(b"sc/inst_idx", le64(idx))
        self._k(b"sc/claimed_sum", running)
        for rd in range(ell_d):
            ys = orc.evals_at(xs)
            s01 = kadd((int(ys[0, 0]), int(ys[0, 1])), (int(ys[1, 0]), int(ys[1, 1])))
            if s01 != (int(running[0]), int(running[1])):
                raise AssertionError(f"ajtai round {rd}: invariant")
            co = interpolate(xs, ys)
            for c in co:
                self._k(b"sumcheck/round/coeff", c)
            r = np.array([tr.challenge_field(b"sumcheck/challenge/0"), tr.challenge_field(b"sumcheck/challenge/1")],
                         np.uint64)
            running = poly_eval_k(co, r)
            orc.fold(r)
            P += [int(v) for v in co.reshape(-1)]
        tr.append_message(b"sc/domain_end", b"ccs/ajtai")
        tr.append_message(b"sc/inst_idx_end", le64(idx))
        P += [int(v) for v in running]
        fold_digest = tr.digest32()
        y_eval, y_sc = orc.me_outputs()        # [k][t][54][2], [k][t][2]
        outs = []
        for i in range(k):
            src = mcs if i == 0 else self.acc[i - 1]
            y = np.zeros((t, d_pad, 2), np.uint64)
            y[:, :D] = y_eval[i]
            outs.append(dict(c=src["c"], X=src["X"], m_in=src["m_in"], r=np.array(r_time), y=y, ysc=y_sc[i],
                             digest=fold_digest))
        P += [int(v) for v in y_eval.reshape(-1)]
        P += [int(v) for v in y_sc.reshape(-1)]
        # Pi_RLC
        tr.append_message(b"fold/rlc_inputs/v1", b"main")
        tr.append_u64s(b"step_idx", [idx])
        tr.append_u64s(b"me_count", [k])
        for me in outs:
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
        A5 = [-2, -1, 0, 1, 2]
        bucket = (1 << 16) // 5 * 5
        rhos = np.zeros((k, D), np.int8)
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
        P += [int(v) % Q for v in rhos.reshape(-1)]
        Zmix = rlc_mix(rhos, Zall, self.threads)
        Rs = [np.eye(D, dtype=np.int64)] if k == 1 else [rot_int(rhos[i]) for i in range(k)]

        def mix_vecs(vecs):  # vecs [k][..][54] ints (F_q) -> sum rot_i vec_i mod q
            acc = None
            for i in range(k):
                v = np.asarray(vecs[i], dtype=object)
                prod = np.tensordot(v, Rs[i].T.astype(object), axes=([-1], [0]))
                acc = prod if acc is None else acc + prod
            return np.vectorize(lambda e: int(e) % Q, otypes=[object])(acc)

        c_parent = mix_vecs([np.asarray(o["c"], np.uint64).astype(object).reshape(kappa, D) for o in outs])
        P += [int(v) for v in c_parent.reshape(-1)]
        y_re = mix_vecs([y_eval[i, :, :, 0].astype(object) for i in range(k)])
        y_im = mix_vecs([y_eval[i, :, :, 1].astype(object) for i in range(k)])
        # Pi_DEC
        planes, nz = split_b(Zmix, self.k_rho, 2)
        ccs_c = [commit_digits(self.pp, planes[i], self.threads).reshape(-1) for i in range(self.k_rho)]
        from . import me_y_at_r
        r_arr = np.array(r_time, np.uint64)
        children, childZ = [], []
        pw = [1]
        for _ in range(1, D):
            pw.append(pw[-1] * 2 % Q)
        ysum_re = np.zeros((t, D), dtype=object)
        ysum_im = np.zeros((t, D), dtype=object)
        csum = np.zeros(kappa * D, dtype=object)
        for i in range(self.k_rho):
            y, ysc = me_y_at_r(self.ccs, planes[i], ell_n, r_arr)
            ypad = np.zeros((t, d_pad, 2), np.uint64)
            ypad[:, :D] = y
            Xc = [int(v) % Q for v in planes[i][:, :m_in].astype(np.int64).reshape(-1)]
            children.append(dict(c=ccs_c[i], X=Xc, m_in=m_in, r=r_arr, y=ypad, ysc=ysc, digest=fold_digest))
            childZ.append(planes[i])
            P += [int(v) for v in ccs_c[i]]
            P += [int(v) for v in y.reshape(-1)]
            ysum_re = ysum_re + (2 ** i) * y[:, :, 0].astype(object)
            ysum_im = ysum_im + (2 ** i) * y[:, :, 1].astype(object)
            csum = csum + (2 ** i) * ccs_c[i].astype(object)
        assert all(int(a) % Q == int(b) for a, b in zip(csum, c_parent.reshape(-1))), "DEC check (c)"
        assert all(int(a) % Q == int(b) for a, b in zip(ysum_re.reshape(-1), y_re.reshape(-1))), "DEC check (y re)"
        assert all(int(a) % Q == int(b) for a, b in zip(ysum_im.reshape(-1), y_im.reshape(-1))), "DEC check (y im)"
        self.acc, self.acc_Z = children, childZ
        self.step_idx += 1
        return np.array(P, dtype=np.uint64)
