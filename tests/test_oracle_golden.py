"""The oracle (oracle/, CPU mpmath restatement) against golden vectors produced by the reference's own code
(tests/golden/make_golden.py): recursion residues, numerator polynomials, pole-shifting columns and the
write_output transforms.  CPU only."""

import mpmath as mp
import pytest

from conftest import golden, golden_operator
from oracle import blocks as OB, derivatives as OD, output as OO, recursion as OR


def _bits(err, scale):
    if err == 0:
        return float("inf")
    return -float(mp.log(err / scale, 2))


@pytest.mark.parametrize("ci", range(4))
def test_recursion_matches_reference_port(ci):
    case = golden("recursion.json")[ci]
    L = case["L"]
    mp.mp.prec = 32 * L + 64
    Mstr, H = golden_operator(case)
    M = {k: [[mp.mpf(x) for x in row] for row in v] for k, v in Mstr.items()}
    pp = tuple(tuple(x) for x in case["pp"])
    worst = mp.inf
    for k in range(case["rhs"]):
        h = {(sp, m, j, a, b): mp.mpf(v) for kk, sp, m, j, a, b, v in H if kk == k}
        res = OR.fill_residues(h, M, case["tj12"], case["tj43"], case["tj_max"], case["order"], pp)
        ref = {tuple(x[1:7]): mp.mpf(x[7]) for x in case["residues"] if x[0] == k}
        assert set(res) == set(ref)
        block = {}
        for key, v in ref.items():
            block[key[:4]] = max(block.get(key[:4], 0), abs(v))
        for key, v in ref.items():
            if block[key[:4]]:
                worst = min(worst, _bits(abs(res[key] - v), block[key[:4]]))
    # the golden residues carry 85 significant digits (~282 bits)
    assert worst > 270, worst


@pytest.mark.parametrize("di", range(2))
def test_numerators_match_reference_port(di):
    d = golden("derivatives.json")[di]
    case = golden("recursion.json")[d["case"]]
    L, R = case["L"], d["R"]
    mp.mp.prec = 32 * L + 64
    hv = {(k, sp, m, j, a, b): mp.mpf(v) for k, sp, m, j, a, b, v in case["h_inf"]}
    rv = {tuple(x[:7]): mp.mpf(x[7]) for x in case["residues"]}
    worst = mp.inf
    for k, tj, p, a, b, e, poly in d["numerators"]:
        h = lambda p_, m, j, a_, b_: hv.get((k, p_, m, j, a_, b_), mp.mpf(0))
        r = lambda p_, m, j, q, a_, b_: rv.get((k, p_, m, j, q, a_, b_), mp.mpf(0))
        got = OD.numerators(h, r, tj, p, a, b, case["order"], R, case["tj12"], case["tj43"])[e]
        ref = [mp.mpf(x) for x in poly]
        assert len(got) == len(ref)
        big = max(abs(x) for x in ref)
        worst = min(worst, _bits(max(abs(x - y) for x, y in zip(got, ref)), big))
    assert worst > 32 * L - 40, worst


@pytest.mark.parametrize("si", range(4))
def test_pole_shifting_solve_matches_closed_form(si):
    """blocks_3d's linear solve (oracle) == the reference's exact closed-form columns, pole by pole"""
    c = golden("shift_columns.json")[si]
    mp.mp.prec = 400
    tj, tj12, tj43, order, kept = c["tj"], c["tj12"], c["tj43"], c["order"], c["kept"]
    ub = mp.mpf(tj) / 2 + (mp.mpf(1) / 2 if tj <= 1 else 1)
    xs = [mp.mpf(OB.twice_pos(P, tj)) / 2 - ub for P in OB.pole_list(tj, tj12, tj43, order)]
    assert [2 * x for x in xs] == [mp.mpf(y) for y in c["roots"]]
    for i, poly, sc, den in c["columns"]:
        unit = [mp.mpf(1) if k == i else mp.mpf(0) for k in range(len(xs))]
        new_x, new_r = OD._shift_poles(xs, unit, tj, tj43, tj12, kept, ub)
        num = [mp.mpf(0)]
        for q, rr in enumerate(new_r):
            num = OD._add(num, [rr * y for y in OD._prod_linear(new_x[:q] + new_x[q + 1:])])
        ref = [mp.mpf(int(v)) / int(den) * mp.mpf(2) ** (k - sc) for k, v in enumerate(poly)]
        ref += [mp.mpf(0)] * (len(num) - len(ref))
        big = max(abs(x) for x in ref) or 1
        assert max(abs(x - y) for x, y in zip(num, ref)) / big < mp.mpf(2) ** -300


@pytest.mark.parametrize("oi", range(5))
def test_write_output_matches_reference(oi):
    c = golden("output.json")[oi]
    mp.mp.prec = 32 * 10 + 128
    Lam, parity, D = c["Lambda"], c["parity"], c["delta_1_plus_2"]
    num = [[mp.mpf(x) for x in row] for row in c["num"]]
    got = OO.xt(num, Lam, parity, D)
    ref = [[mp.mpf(x) for x in row] for row in c["xt"]]
    flat_g = [x for row in got for x in row]
    flat_r = [x for row in ref for x in row]
    big = max(abs(x) for x in flat_r)
    assert _bits(max(abs(a - b) for a, b in zip(flat_g, flat_r)), big) > 270
    T = OO.radial_matrix(Lam, parity, D)
    Tref = c["T_radial"]
    big = max(abs(mp.mpf(x)) for row in Tref for x in row)
    err = max(abs(T[i, j] - mp.mpf(Tref[i][j])) for i in range(len(Tref)) for j in range(len(Tref)))
    assert _bits(err, big) > 270
