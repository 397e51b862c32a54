"""Host-side exact constants of the derivative stages: the pole-shifting numerator columns against the
reference's closed form (derivatives._shift_columns, golden), and the exact polynomial helpers.  CPU only."""
from fractions import Fraction

import pytest

from conftest import golden
from blocksvibe_b200 import derivatives as DV


@pytest.mark.parametrize("si", range(4))
def test_shift_columns_match_reference(si):
    c = golden("shift_columns.json")[si]
    roots, new = c["roots"], c["new"]
    Pi = [1]
    for y0 in new:
        Pi = DV.poly_times_linear(Pi, -y0)
    comp = DV.divide_by_roots(Pi, new)
    cols = DV.shifted_pole_columns(roots, new, comp)
    assert len(cols) == len(c["columns"])
    for (poly, den), (i, rpoly, sc, rden) in zip(cols, c["columns"]):
        mine = [Fraction(v, den) for v in poly]
        ref = [Fraction(int(v), int(rden)) for v in rpoly]
        n = max(len(mine), len(ref))
        mine += [Fraction(0)] * (n - len(mine))
        ref += [Fraction(0)] * (n - len(ref))
        assert mine == ref, i


def test_polynomial_helpers():
    p = [1]
    for r in (-3, 0, 5):
        p = DV.poly_times_linear(p, -r)          # (y + 3) y (y - 5)
    assert p == [0, -15, -2, 1]
    q = DV.divide_by_roots(p, [-3, 0, 5])
    assert q[1] == [-15, -2, 1]
    with pytest.raises(ValueError):
        DV.divide_by_roots(p, [1])
