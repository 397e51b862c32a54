"""Oracle write_output for the xt and xt_radial coordinates, step by step in mpmath: blocks_3d's
lambda_lr_to_lrho_lrhob, congruence_transform with stirling / rho_z / power_prefactor, zzb_to_xt and
lrho_to_xt_radial.  Restates the reference's output.py:35-95 (the transform matrices, blocks_3d's
formulas) and tests/test_blocks_output.py:13-47 (the transforms applied one after the other).
Test infrastructure only."""
import math

import mpmath as mp


def _poch(x, n):
    r = mp.mpf(1)
    for k in range(n):
        r *= x + k
    return r


def falling(x, n):
    """blocks_3d's factorial_power: x (x - 1) ... (x - n + 1), or 1 / ((x + 1) ... (x - n)) for n < 0"""
    return 1 / _poch(x + 1, -n) if n < 0 else _poch(x + 1 - n, n)


def gbinom(k, j):
    """blocks_3d's binomial_coefficient(int k, int j), negative k allowed"""
    if k < j:
        if j < 0:
            return mp.mpf(0)
        num = 1
        for q in range(j):
            num *= k - j + 1 + q
        return mp.mpf(num) / math.factorial(j)
    num = 1
    for q in range(k - j):
        num *= j + 1 + q
    return mp.mpf(num) / math.factorial(k - j)


def stirling(O):
    s = [[mp.mpf(0)] * (O + 1) for _ in range(O + 1)]
    s[0][0] = mp.mpf(1)
    for n in range(O):
        for k in range(n + 1):
            s[n + 1][k + 1] = s[n][k] - n * s[n][k + 1]
    rc = 3 - 2 * mp.sqrt(2)
    return mp.matrix([[s[n][k] / rc ** n for k in range(O + 1)] for n in range(O + 1)])


def rho_z(O):
    z = mp.matrix(O + 1, O + 1)
    r2 = mp.sqrt(2)
    for p in range(O + 1):
        for n in range(p + 1):
            acc = mp.mpf(0)
            for k in range(n + 1):
                acc += (gbinom(n, k) / mp.mpf(2) ** n * (-1) ** k * (4 * r2) ** (n - k) * gbinom(-2 * n, p - k - n)
                        * (4 - 2 * r2) ** (k - n - p))
            z[p, n] = mp.factorial(p) / mp.factorial(n) * acc
    return mp.inverse(z)


def power_prefactor(O, D):
    P = mp.matrix(O + 1, O + 1)
    for n in range(O + 1):
        for k in range(n + 1):
            P[n, k] = falling(-D, n - k) * mp.mpf(2) ** (n - k + D) * gbinom(n, k)
    return P


def one_minus_power_prefactor(O):
    P = mp.matrix(O + 1, O + 1)
    half = mp.mpf(1) / 2
    for n in range(O + 1):
        for k in range(n + 1):
            P[n, k] = (-1) ** (n - k) * falling(-half, n - k) * mp.mpf(2) ** (n - k + half) * gbinom(n, k)
    return P


def congruence(parity, T, tri):
    """Z = T F T^T on the stored triangle j <= min(i, O - i), F(j, i) = (-1)^parity F(i, j)"""
    O = len(tri) - 1
    sym = 1 if parity % 2 == 0 else -1
    inter = [[mp.mpf(0)] * (O + 1) for _ in range(O + 1)]
    for i in range(O + 1):
        for k in range(O + 1):
            for l in range(O + 1 - k):
                f = tri[k][l] if l <= k else sym * tri[l][k]
                inter[i][l] += T[i, k] * f
    return [[mp.fsum(T[j, l] * inter[i][l] for l in range(O)) for j in range(min(i, O - i) + 1)] for i in range(O + 1)]


def xt(num, Lam, parity, delta_1_plus_2):
    """num[idx][e] (lambda order n = parity + 2 idx, log-r derivative e) -> xt[n][b]"""
    O = Lam
    F = [[mp.fsum((-1) ** (j - l) * mp.mpf(2) ** (-i - j) * mp.binomial(i, k) * mp.binomial(j, l)
                  * num[(i + j - k - l - parity) // 2][k + l]
                  for k in range(i + 1) for l in range((i + j - k - parity + 2) % 2, j + 1, 2))
          for j in range(min(i, O - i) + 1)] for i in range(O + 1)]
    Z = congruence(parity, rho_z(O), congruence(parity, stirling(O), F))
    D = mp.mpf(delta_1_plus_2)
    if D != 0:
        Z = congruence(parity, power_prefactor(O, D / 2), Z)
    sym = 1 if parity % 2 == 0 else -1
    out = []
    for n in range(O - parity + 1):
        row = []
        for m in range(parity, O - n + 1, 2):
            r = mp.mpf(0)
            for k in range(n + 1):
                for l in range(m + 1):
                    i, j = n + m - k - l, k + l
                    z = Z[i][j] if i >= j else sym * Z[j][i]
                    r += (-1) ** l * mp.factorial((m - parity) // 2) / mp.factorial(m) * mp.binomial(n, k) \
                        * mp.binomial(m, l) * z
            row.append(r)
        out.append(row)
    return out


def radial_matrix(Lam, parity, delta_1_plus_2):
    O = Lam - parity
    D = mp.mpf(delta_1_plus_2)
    pre = power_prefactor(O, D) if parity == 0 else one_minus_power_prefactor(O) * power_prefactor(O, D + 1)
    return pre * rho_z(O) * stirling(O)


def xt_radial(num0, Lam, parity, delta_1_plus_2):
    """num0[e] (lambda order n = parity) -> xt_radial[i]"""
    T = radial_matrix(Lam, parity, delta_1_plus_2)
    O = Lam - parity
    return [mp.fsum(T[i, j] * num0[j] for j in range(O + 1)) for i in range(O + 1)]
