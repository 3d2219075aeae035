"""Small pure-Python integer restatements used to pin the C oracle.

Written independently of oracle/neo_oracle.c from the definitions:
F_q = Z/qZ, K = F_q[u]/(u^2 - 7), R_q = F_q[X]/(X^54 + X^27 + 1).
"""
Q = (1 << 64) - (1 << 32) + 1
D = 54


def kmul(a, b):
    return ((a[0] * b[0] + 7 * a[1] * b[1]) % Q, (a[0] * b[1] + a[1] * b[0]) % Q)


def poly_mod_phi81(c):
    """Reduce an integer coefficient list modulo X^54 + X^27 + 1 by long division."""
    c = list(c) + [0] * max(0, 2 * D - len(c))
    for i in range(len(c) - 1, D - 1, -1):
        t = c[i]
        if t:
            c[i] = 0
            c[i - D] -= t
            c[i - 27] -= t
    return [x % Q for x in c[:D]]


def rq_mul(a, b):
    prod = [0] * (2 * D - 1)
    for i, x in enumerate(a):
        if x:
            for j, y in enumerate(b):
                prod[i + j] += x * y
    return poly_mod_phi81(prod)


def commit(pp, Z):
    """pp[i][j] = 54 coeffs, Z[r][j] digits -> c[i] = sum_j pp[i][j] * z_j  in R_q."""
    kappa, m = len(pp), len(pp[0])
    out = []
    for i in range(kappa):
        acc = [0] * D
        for j in range(m):
            zj = [int(Z[r][j]) for r in range(D)]
            p = rq_mul([int(x) for x in pp[i][j]], zj)
            acc = [(x + y) % Q for x, y in zip(acc, p)]
        out.append(acc)
    return out


# --- Twist / Shout time-lane sums, dense restatement --------------------------
# Each oracle is a sum over the time hypercube of a product of multilinear
# tables; here every factor is materialised as a dense table (χ_r, eq-bit
# factors, the exclusive prefix sum Val_pre, LT(·, r_time)) and folded on the
# least-significant variable. Independent of the sparse C restatement.

def kadd(a, b):
    return ((a[0] + b[0]) % Q, (a[1] + b[1]) % Q)


def ksub(a, b):
    return ((a[0] - b[0]) % Q, (a[1] - b[1]) % Q)


K0, K1 = (0, 0), (1, 0)


def chi_dense(r):
    t = [K1]
    for ri in r:  # variable i is bit i of the index (little-endian)
        t = [kmul(v, ksub(K1, ri)) for v in t] + [kmul(v, ri) for v in t]
    return t


def eq_bit(bit, u):
    return kadd(kmul(bit, ksub(kadd(u, u), K1)), ksub(K1, u))


def lt_table(r_time):
    ell = len(r_time)
    out = []
    for j in range(1 << ell):
        # LT(j, r) = Σ_i [j_i = 0]·r_i·Π_{k>i} eq(j_k, r_k)
        acc = K0
        for i in range(ell):
            if (j >> i) & 1:
                continue
            term = r_time[i]
            for k in range(i + 1, ell):
                term = kmul(term, r_time[k] if (j >> k) & 1 else ksub(K1, r_time[k]))
            acc = kadd(acc, term)
        out.append(acc)
    return out


def prefix_excl(init, inc_terms):
    out, acc = [], init
    for v in inc_terms:
        out.append(acc)
        acc = kadd(acc, v)
    return out


class DenseMemSum:
    """kind names follow the C ABI: 0 shout value, 1 adapter, 2 bitness,
    3 twist read, 4 twist write, 5 val eval, 6 total inc, 7 product."""

    def __init__(self, kind, cols, r_point=None, r_addr=None, init=K0, weights=None):
        L = len(cols[0])
        A = 0 if r_addr is None else len(r_addr)
        self.kind, self.w = kind, weights
        eqb = lambda col, b: [eq_bit(v, r_addr[b]) for v in col]
        E = chi_dense(r_point) if r_point is not None and kind not in (5,) else None
        if kind == 0:
            F = [E, cols[0], cols[1]]
        elif kind == 1:
            F = [E, cols[0]] + [eqb(cols[1 + b], b) for b in range(A)]
        elif kind == 2:
            F = [E] + list(cols)
        elif kind in (3, 4):
            if kind == 3:
                hw, inc, wa = cols[2 + A], cols[3 + A], cols[4 + A:4 + 2 * A]
            else:
                hw, inc, wa = cols[0], cols[2], cols[3:3 + A]
            terms = []
            for t in range(L):
                v = kmul(hw[t], inc[t])
                for b in range(A):
                    v = kmul(v, eq_bit(wa[b][t], r_addr[b]))
                terms.append(v)
            VP = prefix_excl(init, terms)
            if kind == 3:
                F = [E, cols[0], [ksub(VP[t], cols[1][t]) for t in range(L)]] + [eqb(cols[2 + b], b) for b in range(A)]
            else:
                F = [E, cols[0], [ksub(ksub(cols[1][t], VP[t]), cols[2][t]) for t in range(L)]] + \
                    [eqb(cols[3 + b], b) for b in range(A)]
        elif kind == 5:
            F = [cols[0], cols[1], lt_table(r_point)] + [eqb(cols[2 + b], b) for b in range(A)]
        elif kind == 6:
            F = [cols[0], cols[1]] + [eqb(cols[2 + b], b) for b in range(A)]
        else:
            F = list(cols)
        self.F = [list(f) for f in F]

    def _term(self, vals):
        if self.kind == 2:
            acc = K0
            for w, b in zip(self.w, vals[1:]):
                acc = kadd(acc, kmul(kmul(w, b), ksub(b, K1)))
            return kmul(vals[0], acc)
        p = K1
        for v in vals:
            p = kmul(p, v)
        return p

    def total(self):
        return _ksum(self._term([f[t] for f in self.F]) for t in range(len(self.F[0])))

    def evals(self, xs):
        L = len(self.F[0])
        if L == 1:
            v = self._term([f[0] for f in self.F])
            return [v for _ in xs]
        ys = []
        for x in xs:
            acc = K0
            for p in range(L // 2):
                vals = [kadd(f[2 * p], kmul(ksub(f[2 * p + 1], f[2 * p]), x)) for f in self.F]
                acc = kadd(acc, self._term(vals))
            ys.append(acc)
        return ys

    def fold(self, r):
        if len(self.F[0]) == 1:
            return
        self.F = [[kadd(f[2 * p], kmul(ksub(f[2 * p + 1], f[2 * p]), r)) for p in range(len(f) // 2)] for f in self.F]


def _ksum(it):
    acc = K0
    for v in it:
        acc = kadd(acc, v)
    return acc


class ChaCha8:
    """ChaCha with 8 rounds as a counter-mode u32 stream (RFC 7539 block layout:
    constants, 8 key words, 64-bit block counter in words 12-13, zero nonce)."""

    M = 0xFFFFFFFF

    def __init__(self, seed: bytes):
        assert len(seed) == 32
        self.key = [int.from_bytes(seed[4 * i:4 * i + 4], "little") for i in range(8)]
        self.ctr = 0
        self.buf = []

    @staticmethod
    def _rot(x, n):
        return ((x << n) | (x >> (32 - n))) & ChaCha8.M

    def _block(self):
        s = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + self.key + [self.ctr & self.M, self.ctr >> 32, 0, 0]
        x = list(s)

        def qr(a, b, c, d):
            x[a] = (x[a] + x[b]) & self.M; x[d] = self._rot(x[d] ^ x[a], 16)
            x[c] = (x[c] + x[d]) & self.M; x[b] = self._rot(x[b] ^ x[c], 12)
            x[a] = (x[a] + x[b]) & self.M; x[d] = self._rot(x[d] ^ x[a], 8)
            x[c] = (x[c] + x[d]) & self.M; x[b] = self._rot(x[b] ^ x[c], 7)

        for _ in range(4):
            qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
            qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
        self.ctr += 1
        self.buf = [(a + b) & self.M for a, b in zip(x, s)]

    def next_u32(self):
        if not self.buf:
            self._block()
        return self.buf.pop(0)

    def next_u64(self):
        lo = self.next_u32()
        return lo | (self.next_u32() << 32)

    def fill_bytes(self, n):
        out = b""
        while len(out) < n:
            out += self.next_u32().to_bytes(4, "little")
        return out[:n]


def pp_par_streams(seed: bytes, kappa: int, m: int):
    """setup_par partition: [(chunk seed, first column, columns)] in (row, chunk) order."""
    chunk = max(min(m, 1 << 15), 1024)
    n_chunks = (m + chunk - 1) // chunk
    master = ChaCha8(seed)
    rows = [master.fill_bytes(32) for _ in range(kappa)]
    out = []
    for rs in rows:
        r = ChaCha8(rs)
        for c in range(n_chunks):
            lo = c * chunk
            out.append((r.fill_bytes(32), lo, min(m, lo + chunk) - lo))
    return out
