"""CPU restatement of one Neo fold step, with the shared-CPU-bus memory sidecar.

TEST INFRASTRUCTURE ONLY: the parity checker for neo_gpu_shard_fold_step and
the CPU-baseline leg of bench.py.  It composes the oracle's C primitives in
the order of fold_shard_prove_impl (crates/neo-fold/src/shard.rs:1803-2283)
and prove_rlc_dec_lane (shard.rs:1170-1331), with the transcript calls of
engines/utils.rs:83-212, memory_sidecar/route_a_time.rs:28-152,
memory_sidecar/memory.rs:86-1670 (absorb_step_memory, the Shout/Twist
address pre-time sum-checks, the Route-A time claims, the Twist val-eval
batch and the val-lane CPU ME claims), memory_sidecar/transcript.rs:4-63,
memory_sidecar/sumcheck_ds.rs:11-77 and sumcheck.rs:124-456, and emits the
same canonical step-proof word dump as the CUDA library.
"""
import struct

import numpy as np

from . import (CcsOracle, MemOracle, Transcript, TwistAddrOracle, addr_lookup_weights, bus_openings, ccs_digest,
               commit_digits, decomp_b2, interpolate, me_y_at_r, poly_eval_k, rlc_mix, split_b, u64)

Q = (1 << 64) - (1 << 32) + 1
D = 54


def le64(v):
    return struct.pack("<Q", v)


def kadd(a, b):
    return ((a[0] + b[0]) % Q, (a[1] + b[1]) % Q)


def kmulp(a, b):
    return ((a[0] * b[0] + 7 * a[1] * b[1]) % Q, (a[0] * b[1] + a[1] * b[0]) % Q)


def kt(v):
    return (int(v[0]), int(v[1]))


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


def digest_fields(label, fs):
    """digest_fields (memory_sidecar/transcript.rs:4-10)."""
    h = Transcript(b"memory/public_digest")
    h.append_message(b"digest/label", label)
    h.append_message(b"digest/len", le64(len(fs)))
    h.append_fields(b"digest/fields", [int(v) % Q for v in fs])
    return h.digest32()


def bitness_weights(r0, n, sep):
    """bitness_weights (memory_sidecar/utils.rs:43-71): powers of r_cycle[0] + sep."""
    base = ((int(r0[0]) + sep) % Q, int(r0[1]))
    if base in ((0, 0), (1, 0), (Q - 1, 0)):
        base = ((base[0] + 1) % Q, base[1])
    if base == (0, 0):
        base = (1, 0)
    out, cur = [], (1, 0)
    for _ in range(n):
        out.append(cur)
        cur = kmulp(cur, base)
    return np.array(out, np.uint64).reshape(-1, 2)


class BusLayout:
    """build_bus_layout_for_instances (neo-memory/src/cpu/bus_layout.rs:91-190)."""

    def __init__(self, m, m_in, steps, shout_ell, twist_ell):
        col = 0
        self.shout, self.twist = [], []
        for ea in shout_ell:
            self.shout.append(dict(addr_bits=list(range(col, col + ea)), has_lookup=col + ea, val=col + ea + 1))
            col += ea + 2
        for ea in twist_ell:
            self.twist.append(dict(ra_bits=list(range(col, col + ea)), wa_bits=list(range(col + ea, col + 2 * ea)),
                                   has_read=col + 2 * ea, has_write=col + 2 * ea + 1, wv=col + 2 * ea + 2,
                                   rv=col + 2 * ea + 3, inc=col + 2 * ea + 4))
            col += 2 * ea + 5
        self.bus_cols, self.chunk, self.m_in = col, steps, m_in
        self.bus_base = m - col * steps
        if col and (self.bus_base < m_in):
            raise ValueError("bus region overlaps the public inputs")

    def cell(self, col, j):
        return self.bus_base + col * self.chunk + j


class OracleShard:
    """mem: None (main lane only) or dict(steps=chunk, shout=[dict(ell_addr, k, d, n_side, ell, table)],
    twist=[dict(ell_addr, k, d, n_side, ell, init=[(addr, value)])])."""

    def __init__(self, ccs, pp, m_in=1, k_rho=12, app_label=b"neo/shard", threads=0, mem=None):
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
        self.val_obligations = []
        self.step_idx = 0
        self.threads = threads
        self.mem = mem or dict(steps=0, shout=[], twist=[])
        self.shout = [dict(s) for s in self.mem.get("shout", [])]
        self.twist = [dict(w) for w in self.mem.get("twist", [])]
        self.bus = BusLayout(self.m, m_in, self.mem.get("steps", 0), [s["ell_addr"] for s in self.shout],
                             [w["ell_addr"] for w in self.twist])
        for s in self.shout:
            s["digest"] = digest_fields(b"shout/table", [int(v) for v in s["table"]])
        for w in self.twist:
            init = w.get("init", [])
            if init:
                fs = []
                for a, v in init:
                    fs += [a, v]
                w["digest"] = digest_fields(b"twist/init/sparse", fs)
            else:
                w["digest"] = digest_fields(b"twist/init/zero", [])
        self.prev = None     # previous step's MCS (c, Z) and decoded Twist columns

    def set_twist_init(self, i, init):
        """MemInit of Twist instance i for the following steps (mem_init.rs:26-90):
        [(addr, value)] with strictly increasing addresses, [] = MemInit::Zero."""
        init = [(int(a), int(v) % Q) for a, v in init]
        if any(b[0] <= a[0] for a, b in zip(init, init[1:])):
            raise ValueError("MemInit::Sparse must be strictly increasing by address")
        w = self.twist[i]
        w["init"] = init
        if init:
            fs = []
            for a, v in init:
                fs += [a, v]
            w["digest"] = digest_fields(b"twist/init/sparse", fs)
        else:
            w["digest"] = digest_fields(b"twist/init/zero", [])

    def _k(self, label, v):
        self.tr.append_fields(label, np.array(v, np.uint64))

    def _chal(self, l0=b"batched/challenge/0", l1=b"batched/challenge/1"):
        return np.array([self.tr.challenge_field(l0), self.tr.challenge_field(l1)], np.uint64)

    # ---------------------------------------------------------------- helpers --
    def _time_col(self, zv, col):
        """build_time_sparse_from_bus_col (memory_sidecar/cpu_bus.rs:976-1016), dense."""
        L = 1 << self.ell_n
        out = np.zeros((L, 2), np.uint64)
        for j in range(self.bus.chunk):
            out[self.m_in + j, 0] = zv[self.bus.cell(col, j)]
        return out

    def _bus_y(self, Z, r):
        return bus_openings(Z, self.bus.bus_base, self.bus.chunk, self.bus.bus_cols, self.m_in, np.array(r))

    def _batched(self, claims, n_rounds, P):
        """run_batched_sumcheck_prover (neo-reductions/src/sumcheck.rs:350-456)."""
        tr = self.tr
        running = [kt(c["sum"]) for c in claims]
        chals = []
        for rd in range(n_rounds):
            tr.append_message(b"batched/round_idx", le64(rd))
            polys = []
            for ci, c in enumerate(claims):
                xs = np.array([[x, 0] for x in range(c["deg"] + 1)], np.uint64)
                ys = c["oracle"].evals_at(xs)
                if kadd(kt(ys[0]), kt(ys[1])) != running[ci]:
                    raise AssertionError(f"batched sum-check {c['label']} round {rd}: p(0)+p(1) != running sum")
                polys.append(interpolate(xs, ys))
            for ci, (c, co) in enumerate(zip(claims, polys)):
                tr.append_message(b"batched/claim_label", c["label"])
                tr.append_message(b"batched/claim_idx", le64(ci))
                for coeff in co:
                    self._k(b"batched/round/coeff", coeff)
            r = self._chal()
            chals.append(r)
            for ci, (c, co) in enumerate(zip(claims, polys)):
                running[ci] = kt(poly_eval_k(co, r))
                c["oracle"].fold(r)
                P += [int(v) for v in co.reshape(-1)]
        return chals, running

    def _batched_ds(self, domain, inst_idx, claims, n_rounds, P):
        self.tr.append_message(b"sc/domain", domain)
        self.tr.append_message(b"sc/inst_idx", le64(inst_idx))
        out = self._batched(claims, n_rounds, P)
        self.tr.append_message(b"sc/domain_end", domain)
        self.tr.append_message(b"sc/inst_idx_end", le64(inst_idx))
        return out

    def _bind_claim_sums(self, prefix, sums, labels):
        """bind_batched_claim_sums (memory_sidecar/transcript.rs:12-26)."""
        self.tr.append_message(prefix, le64(len(sums)))
        for i, (s, lab) in enumerate(zip(sums, labels)):
            self.tr.append_message(b"addr_batch/label", lab)
            self.tr.append_message(b"addr_batch/idx", le64(i))
            self._k(b"addr_batch/claimed_sum", s)

    def _sample_ext_point(self, label, l0, l1, n):
        out = []
        for i in range(n):
            self.tr.append_message(label, le64(i))
            out.append(np.array([self.tr.challenge_field(l0), self.tr.challenge_field(l1)], np.uint64))
        return out

    def _rlc_dec_lane(self, lane, idx, ins, wits, r, fold_digest, P):
        """prove_rlc_dec_lane (shard.rs:1170-1331) with bus openings for the children."""
        tr, t, kappa, m_in = self.tr, self.t, self.kappa, self.m_in
        k = len(ins)
        d_pad = 1 << self.ell_d
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
        Zall = np.stack(wits)
        Zmix = rlc_mix(rhos, Zall, self.threads)
        Rs = [np.eye(D, dtype=np.int64)] if k == 1 else [rot_int(rhos[i]) for i in range(k)]

        def mix_vecs(vecs):  # vecs [k][..][54] ints (F_q) -> sum rot_i vec_i mod q
            acc = None
            for i in range(k):
                v = np.asarray(vecs[i], dtype=object)
                prod = np.tensordot(v, Rs[i].T.astype(object), axes=([-1], [0]))
                acc = prod if acc is None else acc + prod
            return np.vectorize(lambda e: int(e) % Q, otypes=[object])(acc)

        c_parent = mix_vecs([np.asarray(o["c"], np.uint64).astype(object).reshape(kappa, D) for o in ins])
        P += [int(v) for v in c_parent.reshape(-1)]
        ycore = [np.asarray(o["y"], np.uint64)[:t, :D] for o in ins]
        y_re = mix_vecs([y[:, :, 0].astype(object) for y in ycore])
        y_im = mix_vecs([y[:, :, 1].astype(object) for y in ycore])
        planes, nz = split_b(Zmix, self.k_rho, 2)
        ccs_c = [commit_digits(self.pp, planes[i], self.threads).reshape(-1) for i in range(self.k_rho)]
        r_arr = np.array(r, np.uint64)
        children, childZ = [], []
        ysum_re = np.zeros((t, D), dtype=object)
        ysum_im = np.zeros((t, D), dtype=object)
        csum = np.zeros(kappa * D, dtype=object)
        nb = self.bus.bus_cols
        for i in range(self.k_rho):
            y, ysc = me_y_at_r(self.ccs, planes[i], self.ell_n, r_arr)
            ypad = np.zeros((t + nb, d_pad, 2), np.uint64)
            ypad[:t, :D] = y
            ysc_all = np.zeros((t + nb, 2), np.uint64)
            ysc_all[:t] = ysc
            if nb:
                by, bsc = self._bus_y(planes[i], r)
                ypad[t:, :D] = by
                ysc_all[t:] = bsc
            Xc = [int(v) % Q for v in planes[i][:, :m_in].astype(np.int64).reshape(-1)]
            children.append(dict(c=ccs_c[i], X=Xc, m_in=m_in, r=r_arr, y=ypad, ysc=ysc_all, digest=fold_digest))
            childZ.append(planes[i])
            P += [int(v) for v in ccs_c[i]]
            P += [int(v) for v in y.reshape(-1)]
            if nb:
                P += [int(v) for v in ypad[t:, :D].reshape(-1)]
            ysum_re = ysum_re + (2 ** i) * y[:, :, 0].astype(object)
            ysum_im = ysum_im + (2 ** i) * y[:, :, 1].astype(object)
            csum = csum + (2 ** i) * ccs_c[i].astype(object)
        assert all(int(a) % Q == int(b) for a, b in zip(csum, c_parent.reshape(-1))), "DEC check (c)"
        assert all(int(a) % Q == int(b) for a, b in zip(ysum_re.reshape(-1), y_re.reshape(-1))), "DEC check (y re)"
        assert all(int(a) % Q == int(b) for a, b in zip(ysum_im.reshape(-1), y_im.reshape(-1))), "DEC check (y im)"
        return children, childZ

    # -------------------------------------------------------------- fold step --
    def fold_step(self, z):
        tr, t, ell_n, ell_d, d_sc = self.tr, self.t, self.ell_n, self.ell_d, self.d_sc
        idx, kappa, m_in = self.step_idx, self.kappa, self.m_in
        bus, nb = self.bus, self.bus.bus_cols
        n_acc = len(self.acc)
        k = 1 + n_acc
        d_pad = 1 << ell_d
        P = []
        zv = [int(v) % Q for v in np.asarray(z, np.uint64)]
        Zm = decomp_b2(z)
        c_mcs = commit_digits(self.pp, Zm, self.threads).reshape(-1)
        P += [int(v) for v in c_mcs]
        x = zv[:m_in]
        Xm = [int(v) % Q for v in Zm[:, :m_in].astype(np.int64).reshape(-1)]
        mcs = dict(c=c_mcs, X=Xm, m_in=m_in)
        # absorb_step_memory (memory_sidecar/memory.rs:86-124)
        tr.append_message(b"step/absorb_memory_start")
        tr.append_message(b"step/lut_count", le64(len(self.shout)))
        for i, s in enumerate(self.shout):
            tr.append_message(b"step/lut_idx", le64(i))
            tr.append_message(b"shout/k", le64(s["k"]))
            tr.append_message(b"shout/d", le64(s["d"]))
            tr.append_message(b"shout/n_side", le64(s["n_side"]))
            tr.append_message(b"shout/steps", le64(bus.chunk))
            tr.append_message(b"shout/ell", le64(s["ell"]))
            tr.append_message(b"shout/table_digest", s["digest"])
        tr.append_message(b"step/mem_count", le64(len(self.twist)))
        for i, w in enumerate(self.twist):
            tr.append_message(b"step/mem_idx", le64(i))
            tr.append_message(b"twist/k", le64(w["k"]))
            tr.append_message(b"twist/d", le64(w["d"]))
            tr.append_message(b"twist/n_side", le64(w["n_side"]))
            tr.append_message(b"twist/steps", le64(bus.chunk))
            tr.append_message(b"twist/ell", le64(w["ell"]))
            tr.append_message(b"twist/init_digest", w["digest"])
        tr.append_message(b"step/absorb_memory_done")
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
        # claimed_initial_sum_from_inputs (core rows only)
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
                        ye = kadd(ye, kmulp(kt(me["y"][j][rho]), chi_a[rho]))
                    inner = kadd(inner, kmulp(kmulp(gi, gkj), ye))
                gkj = kmulp(gkj, gk)
            T = kmulp(gk, inner)
        self._k(b"sumcheck/initial_sum", T)
        P += list(T)
        r_cycle = self._sample_ext_point(b"route_a/r_cycle", b"route_a/cycle/0", b"route_a/cycle/1", ell_n)
        r_cyc = np.array(r_cycle)
        # CCS oracle
        Zall = np.stack([Zm] + self.acc_Z)
        rin = np.array(self.acc[0]["r"], np.uint64) if n_acc else None
        orc = CcsOracle(self.ccs, Zall, 2, np.array(alpha, np.uint64), np.array(beta_a, np.uint64),
                        np.array(beta_r, np.uint64), np.array(gamma, np.uint64), rin, ell_d, ell_n, d_sc)
        # ---- memory: decode the bus columns of this step ----
        col = lambda c: self._time_col(zv, c)
        shout_dec = [dict(addr_bits=np.stack([col(c) for c in sc["addr_bits"]]), has=col(sc["has_lookup"]),
                          val=col(sc["val"])) for sc in bus.shout]
        twist_dec = [dict(ra=np.stack([col(c) for c in tc["ra_bits"]]), wa=np.stack([col(c) for c in tc["wa_bits"]]),
                          hr=col(tc["has_read"]), hw=col(tc["has_write"]), wv=col(tc["wv"]), rv=col(tc["rv"]),
                          inc=col(tc["inc"])) for tc in bus.twist]
        # ---- Shout address pre-time (memory.rs:430-621) ----
        r_addr_s = []
        if self.shout:
            ea = self.shout[0]["ell_addr"]
            sums, active, orcs = [], 0, []
            for i, (s, dcd) in enumerate(zip(self.shout, shout_dec)):
                if any(dcd["has"][:, 0]) or any(dcd["has"][:, 1]):
                    tab = np.zeros((len(s["table"]), 2), np.uint64)
                    tab[:, 0] = np.asarray(s["table"], np.uint64) % np.uint64(Q)
                    w, cl = addr_lookup_weights(r_cyc, dcd["has"], dcd["addr_bits"], tab)
                    tk = np.zeros((1 << ea, 2), np.uint64)
                    n_t = min(len(tab), 1 << ea)
                    tk[:n_t] = tab[:n_t]
                    orcs.append(dict(oracle=MemOracle(7, np.stack([tk, w])), sum=cl, label=b"shout/addr_pre", deg=2))
                    sums.append(cl)
                    active |= 1 << i
                else:
                    sums.append(np.zeros(2, np.uint64))
            tr.append_message(b"shout/addr_pre_time/step_idx", le64(idx))
            self._bind_claim_sums(b"shout/addr_pre_time/claimed_sums", sums, [b"shout/addr_pre"] * len(sums))
            for s in sums:
                P += [int(v) for v in s]
            P.append(active)
            if active == 0:
                tr.append_message(b"shout/addr_pre_time/no_sumcheck", le64(idx))
                r_addr_s = self._sample_ext_point(b"shout/addr_pre_time/no_sumcheck/r_addr",
                                                  b"shout/addr_pre_time/no_sumcheck/r_addr/0",
                                                  b"shout/addr_pre_time/no_sumcheck/r_addr/1", ea)
            else:
                r_addr_s, _ = self._batched_ds(b"shout/addr_pre_time", idx, orcs, ea, P)
            for r in r_addr_s:
                P += [int(v) for v in r]
        # ---- Twist address pre-time (memory.rs:232-428) ----
        twist_pre = []
        for i, (w, dcd) in enumerate(zip(self.twist, twist_dec)):
            ea = w["ell_addr"]
            init = [(a, (v % Q, 0)) for a, v in w.get("init", [])]
            rcols = np.concatenate([dcd["hr"][None], dcd["rv"][None], dcd["ra"], dcd["hw"][None], dcd["inc"][None],
                                    dcd["wa"]])
            wcols = np.concatenate([dcd["hw"][None], dcd["wv"][None], dcd["inc"][None], dcd["wa"]])
            ro = TwistAddrOracle(0, rcols, r_cyc, ea, init)
            wo = TwistAddrOracle(1, wcols, r_cyc, ea, init)
            labels = [b"twist/read_addr_pre", b"twist/write_addr_pre"]
            tr.append_message(b"twist/addr_pre_time/claim_idx", le64(i))
            zero = np.zeros(2, np.uint64)
            self._bind_claim_sums(b"twist/addr_pre_time/claimed_sums", [zero, zero], labels)
            claims = [dict(oracle=ro, sum=zero, label=labels[0], deg=2), dict(oracle=wo, sum=zero, label=labels[1], deg=2)]
            r_addr, fin = self._batched_ds(b"twist/addr_pre_time", i, claims, ea, P)
            for r in r_addr:
                P += [int(v) for v in r]
            P += list(fin[0]) + list(fin[1])
            twist_pre.append(dict(r_addr=r_addr, read=fin[0], write=fin[1], rcols=rcols, wcols=wcols))
        # ---- Route-A time claims (memory.rs:905-1033) + batched time sum-check (route_a_time.rs:28-152) ----
        claims = [dict(oracle=orc, sum=np.array(T, np.uint64), label=b"ccs/time", deg=d_sc, dyn=True)]
        for i, (s, dcd) in enumerate(zip(self.shout, shout_dec)):
            ea = s["ell_addr"]
            v = MemOracle(0, np.stack([dcd["has"], dcd["val"]]), r_cyc)
            a = MemOracle(1, np.concatenate([dcd["has"][None], dcd["addr_bits"]]), r_cyc, np.array(r_addr_s))
            bcols = np.concatenate([dcd["addr_bits"], dcd["has"][None]])
            bw = bitness_weights(r_cycle[0], bcols.shape[0], 0x5348_4F55_54 + i)
            bo = MemOracle(2, bcols, r_cyc, weights=bw)
            claims += [dict(oracle=v, sum=v.claim, label=b"shout/value", deg=3, dyn=True),
                       dict(oracle=a, sum=a.claim, label=b"shout/adapter", deg=2 + ea, dyn=True),
                       dict(oracle=bo, sum=np.zeros(2, np.uint64), label=b"shout/bitness", deg=3, dyn=False)]
        for i, (w, dcd, pre) in enumerate(zip(self.twist, twist_dec, twist_pre)):
            ea = w["ell_addr"]
            init_r = (0, 0)
            for a_, v_ in w.get("init", []):
                chi = (1, 0)
                for bit, rb in enumerate(pre["r_addr"]):
                    rb = kt(rb)
                    chi = kmulp(chi, rb if (a_ >> bit) & 1 else ((1 - rb[0]) % Q, (-rb[1]) % Q))
                init_r = kadd(init_r, kmulp((v_ % Q, 0), chi))
            init_r = np.array(init_r, np.uint64)
            ro = MemOracle(3, pre["rcols"], r_cyc, np.array(pre["r_addr"]), init_r)
            wo = MemOracle(4, pre["wcols"], r_cyc, np.array(pre["r_addr"]), init_r)
            bcols = np.concatenate([dcd["ra"], dcd["wa"], dcd["hr"][None], dcd["hw"][None]])
            bw = bitness_weights(r_cycle[0], bcols.shape[0], 0x5457_4953_54 + i)
            bo = MemOracle(2, bcols, r_cyc, weights=bw)
            claims += [dict(oracle=ro, sum=np.array(pre["read"], np.uint64), label=b"twist/read_check", deg=3 + ea,
                            dyn=True),
                       dict(oracle=wo, sum=np.array(pre["write"], np.uint64), label=b"twist/write_check", deg=3 + ea,
                            dyn=True),
                       dict(oracle=bo, sum=np.zeros(2, np.uint64), label=b"twist/bitness", deg=3, dyn=False)]
        # bind_batched_dynamic_claims (memory_sidecar/transcript.rs:37-63)
        tr.append_message(b"batched/dynamic_bind/len", le64(len(claims)))
        for ci, c in enumerate(claims):
            tr.append_message(b"batched/dynamic_bind/claim_label", c["label"])
            tr.append_message(b"batched/dynamic_bind/claim_idx", le64(ci))
            tr.append_message(b"batched/dynamic_bind/degree_bound", le64(c["deg"]))
            tr.append_message(b"batched/dynamic_bind/is_dynamic", bytes([1 if c["dyn"] else 0]))
            if c["dyn"]:
                self._k(b"batched/dynamic_bind/claimed_sum", c["sum"])
        r_time, finals = self._batched_ds(b"shard/batched_time", idx, claims, ell_n, P)
        running = np.array(finals[0], np.uint64)
        # Ajtai rounds
        xs = np.array([[i, 0] for i in range(d_sc + 1)], np.uint64)
        tr.append_message(b"sc/domain", b"ccs/ajtai")
        tr.append_message(b"sc/inst_idx", le64(idx))
        self._k(b"sc/claimed_sum", running)
        for rd in range(ell_d):
            ys = orc.evals_at(xs)
            if kadd(kt(ys[0]), kt(ys[1])) != kt(running):
                raise AssertionError(f"ajtai round {rd}: invariant")
            co = interpolate(xs, ys)
            for c in co:
                self._k(b"sumcheck/round/coeff", c)
            r = self._chal(b"sumcheck/challenge/0", b"sumcheck/challenge/1")
            running = poly_eval_k(co, r)
            orc.fold(r)
            P += [int(v) for v in co.reshape(-1)]
        tr.append_message(b"sc/domain_end", b"ccs/ajtai")
        tr.append_message(b"sc/inst_idx_end", le64(idx))
        P += [int(v) for v in running]
        fold_digest = tr.digest32()
        y_eval, y_sc = orc.me_outputs()        # [k][t][54][2], [k][t][2]
        outs_Z = [Zm] + self.acc_Z
        outs = []
        bus_ys = []
        for i in range(k):
            src = mcs if i == 0 else self.acc[i - 1]
            y = np.zeros((t + nb, d_pad, 2), np.uint64)
            y[:t, :D] = y_eval[i]
            ysc = np.zeros((t + nb, 2), np.uint64)
            ysc[:t] = y_sc[i]
            if nb:
                by, bsc = self._bus_y(outs_Z[i], r_time)
                y[t:, :D] = by
                ysc[t:] = bsc
                bus_ys.append(y[t:, :D])
            outs.append(dict(c=src["c"], X=src["X"], m_in=src["m_in"], r=np.array(r_time), y=y, ysc=ysc,
                             digest=fold_digest))
        P += [int(v) for v in y_eval.reshape(-1)]
        P += [int(v) for v in y_sc.reshape(-1)]
        for i in range(len(bus_ys)):
            P += [int(v) for v in bus_ys[i].reshape(-1)] + [int(v) for v in outs[i]["ysc"][t:].reshape(-1)]
        # ---- finalize_route_a_memory_prover (memory.rs:1284-1670) ----
        val_claims, val_wits = [], []
        has_prev = self.prev is not None
        if self.twist:
            vcl = []
            for i, (w, pre) in enumerate(zip(self.twist, twist_pre)):
                ea = w["ell_addr"]
                dcd = twist_dec[i]
                vcols = np.concatenate([dcd["hw"][None], dcd["inc"][None], dcd["wa"]])
                lt = MemOracle(5, vcols, np.array(r_time), np.array(pre["r_addr"]))
                tot = MemOracle(6, vcols, None, np.array(pre["r_addr"]))
                vcl += [dict(oracle=lt, sum=lt.claim, label=b"twist/val_eval_lt", deg=ea + 3, tag=0),
                        dict(oracle=tot, sum=tot.claim, label=b"twist/val_eval_total", deg=ea + 2, tag=1)]
                if has_prev:
                    pd = self.prev["twist_dec"][i]
                    pcols = np.concatenate([pd["hw"][None], pd["inc"][None], pd["wa"]])
                    pt = MemOracle(6, pcols, None, np.array(pre["r_addr"]))
                    vcl.append(dict(oracle=pt, sum=pt.claim, label=b"twist/rollover_prev_total", deg=ea + 2, tag=2))
            tr.append_message(b"twist/val_eval/batch_start", le64(len(self.twist)))
            tr.append_message(b"twist/val_eval/step_idx", le64(idx))
            tr.append_message(b"twist/val_eval/claimed_sums_len", le64(len(vcl)))
            for ci, c in enumerate(vcl):
                tr.append_message(b"twist/val_eval/claim_idx", le64(ci))
                tr.append_message(b"twist/val_eval/claim_kind", bytes([c["tag"]]))
                self._k(b"twist/val_eval/claimed_sum", c["sum"])
                P += [int(v) for v in c["sum"]]
            r_val, _ = self._batched_ds(b"twist/val_eval_batch", idx, vcl, ell_n, P)
            tr.append_message(b"twist/val_eval/batch_done")
            for r in r_val:
                P += [int(v) for v in r]
            # CPU ME claims at r_val (ts_common.rs:100-258) with bus openings
            fork = tr.clone_state()
            fork.append_message(b"fork", b"cpu_bus/me_digest_val")
            vdigest = fork.digest32()
            srcs = [(c_mcs, Zm, Xm)]
            if has_prev:
                srcs.append((self.prev["c"], self.prev["Z"], self.prev["X"]))
            rv_arr = np.array(r_val, np.uint64)
            for c_, Z_, X_ in srcs:
                yv, yvs = me_y_at_r(self.ccs, Z_, ell_n, rv_arr)
                y = np.zeros((t + nb, d_pad, 2), np.uint64)
                y[:t, :D] = yv
                ysc = np.zeros((t + nb, 2), np.uint64)
                ysc[:t] = yvs
                by, bsc = self._bus_y(Z_, r_val)
                y[t:, :D] = by
                ysc[t:] = bsc
                val_claims.append(dict(c=c_, X=X_, m_in=m_in, r=rv_arr, y=y, ysc=ysc, digest=vdigest))
                val_wits.append(Z_)
                P += [int(v) for v in y[:, :D].reshape(-1)] + [int(v) for v in ysc.reshape(-1)]
        # ---- main lane ----
        children, childZ = self._rlc_dec_lane(b"main", idx, outs, outs_Z, r_time, fold_digest, P)
        # ---- val lane ----
        if val_claims:
            tr.append_message(b"fold/val_lane_start", le64(idx))
            vch, _ = self._rlc_dec_lane(b"val", idx, val_claims, val_wits, r_val, vdigest, P)
            self.val_obligations += vch
        tr.append_message(b"fold/step_done", le64(idx))
        self.acc, self.acc_Z = children, childZ
        if self.twist:
            self.prev = dict(c=c_mcs, Z=Zm, X=Xm, twist_dec=twist_dec)
        self.step_idx += 1
        return np.array(P, dtype=np.uint64)
