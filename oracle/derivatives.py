"""Oracle post-recursion stages, in mpmath, for one (spin, parity, structure, right-hand side):
blocks_3d's residues_to_derivatives, restore_r_delta (division of each pole's polynomial by Delta - D_i),
shift_fraction (Delta -> x + ub) and together_with_factors, restating the reference's mpmath port
tests/test_blocks_derivatives.py:36-80; plus blocks_3d's pole shifting done the way blocks_3d does it,
by solving A a' = V a (the reference describes it in derivatives.py:27-33 and replaces it by a closed
form).  Test infrastructure only.

Polynomials are lists of coefficients, lowest degree first.
"""
from math import comb

import mpmath as mp

from . import blocks as B


def _mul(p, q):
    out = [mp.mpf(0)] * (len(p) + len(q) - 1)
    for i, x in enumerate(p):
        for j, y in enumerate(q):
            out[i + j] += x * y
    return out


def _add(p, q):
    n = max(len(p), len(q))
    return [(p[i] if i < len(p) else 0) + (q[i] if i < len(q) else 0) for i in range(n)]


def _div_linear(p, r):
    """p(x) = (x - r) q(x) + rem"""
    q = [mp.mpf(0)] * max(len(p) - 1, 0)
    acc = mp.mpf(0)
    for k in range(len(p) - 1, 0, -1):
        acc = p[k] + r * acc
        q[k - 1] = acc
    return q, (p[0] + r * acc if p else mp.mpf(0))


def _prod_linear(roots):
    out = [mp.mpf(1)]
    for x in roots:
        out = _mul(out, [-x, mp.mpf(1)])
    return out


def numerators(h, res, tj, p, a, b, order, R, tj12, tj43, kept_pole_order=None):
    """numerator polynomials num_e(x), e = 0..R, of one block.  h(p, m, jh, a, b) and
    res(p, m, jidx, pole index, a, b) return numbers (zero where absent)."""
    rc = 3 - 2 * mp.sqrt(2)
    w = [[(mp.mpf(n) ** k if (n or k) else mp.mpf(1)) * rc ** n for n in range(order + 1)] for k in range(R + 1)]
    jh = (tj - tj12 % 2) // 2
    c = [mp.fsum(w[k][m] * h(p, m, jh, a, b) for m in range(order + 1)) for k in range(R + 1)]
    poles = []
    for P in B.pole_list(tj, tj12, tj43, order):
        s = B.shift(P)
        v = [mp.fsum(w[k][m + s] * res(p, m, jh, B.pole_list(tj, tj12, tj43, order - m).index(P), a, b)
                     for m in range(order - s + 1)) for k in range(R + 1)]
        poles.append((mp.mpf(B.twice_pos(P, tj)) / 2, v))
    ub = mp.mpf(tj) / 2 + (mp.mpf(1) / 2 if tj <= 1 else 1)
    xs = [D - ub for D, _ in poles]

    def binom_power(e, d):                        # C(e, d) Delta^(e - d) as a polynomial in Delta
        return [mp.mpf(0)] * (e - d) + [mp.mpf(comb(e, d))] if d <= e else [mp.mpf(0)]

    out = []
    for e in range(R + 1):
        poly = [mp.mpf(0)]
        for d in range(R + 1):
            poly = _add(poly, [t * c[d] for t in binom_power(e, d)])
        resid = []
        for D, v in poles:
            part = [mp.mpf(0)]
            for d in range(R + 1):
                part = _add(part, [t * v[d] for t in binom_power(e, d)])
            q, rem = _div_linear(part, D)
            poly = _add(poly, q)
            resid.append(rem)
        shifted, power = [mp.mpf(0)], [mp.mpf(1)]  # poly(x + ub)
        for t in poly:
            shifted = _add(shifted, [t * y for y in power])
            power = _mul(power, [ub, mp.mpf(1)])
        if kept_pole_order is None or kept_pole_order >= order:
            new_poles, new_resid = xs, resid
        else:
            new_poles, new_resid = _shift_poles(xs, resid, tj, tj43, tj12, kept_pole_order, ub)
        num = _mul(shifted, _prod_linear(new_poles))
        for i, r in enumerate(new_resid):
            num = _add(num, [r * y for y in _prod_linear(new_poles[:i] + new_poles[i + 1:])])
        out.append(num)
    return out


def _shift_poles(xs, resid, tj, tj43, tj12, kept_pole_order, ub):
    """blocks_3d's pole shifting: keep the protected poles (x = 0) with their residues; replace the others
    by the poles of the block at kept_pole_order (x != 0) with residues a' = A^-1 V a,
    A[r][k] = keep_k^(r - h), V[r][i] = x_i^(r - h), r < size, h = size // 2."""
    prot = [(x, r) for x, r in zip(xs, resid) if x == 0]
    unprot = [(x, r) for x, r in zip(xs, resid) if x != 0]
    keep = [mp.mpf(B.twice_pos(P, tj)) / 2 - ub for P in B.pole_list(tj, tj12, tj43, kept_pole_order)]
    keep = [x for x in keep if x != 0]
    size = len(keep)
    if size == 0:
        return [x for x, _ in prot], [r for _, r in prot]
    h = size // 2
    A = mp.matrix(size, size)
    V = mp.matrix(size, len(unprot))
    for r in range(size):
        for k in range(size):
            A[r, k] = keep[k] ** (r - h)
        for i, (x, _) in enumerate(unprot):
            V[r, i] = x ** (r - h)
    a = mp.matrix([r for _, r in unprot]) if unprot else mp.matrix(0, 1)
    rhs = V * a if unprot else mp.matrix([0] * size)
    shifted = mp.lu_solve(A, rhs)
    return [x for x, _ in prot] + keep, [r for _, r in prot] + [shifted[k] for k in range(size)]
