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
