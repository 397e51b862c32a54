"""Host-side exact constants of the derivative stages: the numerator basis with pole shifting against the
reference's own pole-shifting columns (derivatives._shift_columns, golden), and against blocks_3d's definition
of pole shifting (a linear solve A a' = V a) done here with exact rationals.  CPU only."""
from fractions import Fraction

import pytest

from conftest import golden
from blocksvibe_b200 import derivatives as DV, structure as S


def _pad(p, n):
    return list(p) + [Fraction(0)] * (n - len(p))


@pytest.mark.parametrize("si", range(4))
def test_pole_columns_match_reference(si):
    c = golden("shift_columns.json")[si]
    tj, tj12, tj43, order, kept = (int(c[k]) for k in ("tj", "tj12", "tj43", "order", "kept"))
    poles, _, npj = DV.numerator_basis_y(tj, tj12, tj43, order, kept)
    assert npj == len(c["new"])
    assert len(poles) == len(c["columns"]) == len(c["roots"])
    for mine, (i, rpoly, sc, rden) in zip(poles, c["columns"]):
        ref = [Fraction(int(v), int(rden)) for v in rpoly]
        n = max(len(mine), len(ref))
        assert _pad(mine, n) == _pad(ref, n), i
        assert sc == npj - 1


def _solve(A, b):
    """exact Gaussian elimination"""
    n = len(A)
    M = [row[:] + [v] for row, v in zip(A, b)]
    for c in range(n):
        piv = next(r for r in range(c, n) if M[r][c] != 0)
        M[c], M[piv] = M[piv], M[c]
        for r in range(n):
            if r != c and M[r][c] != 0:
                f = M[r][c] / M[c][c]
                M[r] = [x - f * y for x, y in zip(M[r], M[c])]
    return [M[r][n] / M[r][r] for r in range(n)]


@pytest.mark.parametrize("tj,tj12,tj43,order,kept", [(4, 2, 2, 7, 4), (0, 0, 0, 10, 6), (6, 8, 8, 12, 5), (3, 1, 1, 9, 4)])
def test_shifted_columns_are_blocks3d_pole_shifting(tj, tj12, tj43, order, kept):
    """sum_i a_i column_i(y) = sum over protected poles a_p Pi / y + sum_k a'_k Pi / (y - y'_k), a' = A^-1 V a
    (A[r][k] = y'_k^(r - h), V[r][i] = y_i^(r - h), r < #kept, h = #kept // 2): checked per unit residue a = e_i"""
    two_ub = tj + 1 if tj <= 1 else tj + 2
    ys = [S.twice_position(P, tj) - two_ub for P in S.block_poles(tj, tj12, tj43, order)]
    keep = [y for y in (S.twice_position(P, tj) - two_ub for P in S.block_poles(tj, tj12, tj43, kept)) if y != 0]
    poles, polys, npj = DV.numerator_basis_y(tj, tj12, tj43, order, kept)
    Pi = polys[0]
    assert npj == ys.count(0) + len(keep) and len(Pi) == npj + 1
    h = len(keep) // 2
    A = [[Fraction(y) ** (r - h) for y in keep] for r in range(len(keep))]
    for yi, col in zip(ys, poles):
        if yi == 0:
            want, _ = DV._deflate(Pi, 0)
        else:
            a2 = _solve(A, [Fraction(yi) ** (r - h) for r in range(len(keep))])
            want = [Fraction(0)] * npj
            for ak, yk in zip(a2, keep):
                q, rem = DV._deflate(Pi, yk)
                assert rem == 0
                want = [w + ak * v for w, v in zip(want, q)]
        n = max(len(col), len(want))
        assert _pad(col, n) == _pad(want, n), yi


def test_unshifted_columns_divide_pi():
    """without pole shifting: pole column i = Pi / (y - y_i), polynomial column t = Pi (y + 2 ub)^t"""
    tj, two_ub = 4, 6
    poles, polys, npj = DV.numerator_basis_y(tj, 2, 2, 6, None, R=2)
    Pi = polys[0]
    ys = [S.twice_position(P, tj) - two_ub for P in S.block_poles(tj, 2, 2, 6)]
    assert npj == len(ys) == len(Pi) - 1
    for yi, col in zip(ys, poles):
        q, rem = DV._deflate(Pi, yi)
        assert rem == 0 and col == q
    for t in (1, 2):
        prev = polys[t - 1]
        assert polys[t] == [two_ub * prev[0]] + [prev[k - 1] + two_ub * prev[k] for k in range(1, len(prev))] + [prev[-1]]
