"""The JSON-output oracle (oracle/jsonfmt.py) and the host half of the GPU writer (blocksvibe_b200/jsonout.py:
header, digit counts) against the reference writer's own output (tests/golden/json_output.json, made by
b3djson.fmt_big / write_spin on the seeded values of tests/golden/json_cases.py).  CPU only."""
import os
import sys
from decimal import Decimal, ROUND_HALF_EVEN, localcontext

import pytest

from conftest import GOLDEN, golden
from blocksvibe_b200 import jsonout as JO
from oracle import jsonfmt as OJ

sys.path.insert(0, GOLDEN)
import json_cases as JC  # noqa: E402


def test_digits10_matches_reference_table():
    assert [JO.digits10(b) for b in (256, 512, 768, 896, 1024, 1280)] == [77, 154, 231, 269, 308, 385]
    assert [OJ.digits10(b) for b in (256, 1024, 1280)] == [77, 308, 385]


@pytest.mark.parametrize("ci", range(len(JC.NUMBER_CASES)))
def test_oracle_numbers_match_reference(ci):
    g = golden("json_output.json")["numbers"][ci]
    vals = JC.random_numbers(g["L"], g["count"], g["seed"])
    got = [OJ.fmt(v, e, g["p"]) for v, e in vals]
    assert got == g["text"]


def test_oracle_rounds_ties_to_even():
    """MPFR's round-to-nearest (the production writer): exact halves go to the even neighbour"""
    assert OJ.fmt(125, 0, 2) == "1.2e+02" and OJ.fmt(135, 0, 2) == "1.4e+02"
    assert OJ.fmt(-25, -1, 1) == "-1e+01" and OJ.fmt(-5, -1, 1) == "-2" and OJ.fmt(5, -1, 1) == "2" and OJ.fmt(15, -1, 1) == "8"
    p = 40
    for v, e in [((1 << 140) + 1, -140), (3 * (1 << 139) + 1, -139), ((5 << 200) + 1, -200)]:
        with localcontext() as ctx:
            ctx.prec = 400
            x = Decimal(v) / Decimal(2) ** -e
            E = x.adjusted()
            q = x.scaleb(p - 1 - E).quantize(Decimal(1), rounding=ROUND_HALF_EVEN)
        digs, E2 = OJ.decimal_digits(v, e, p)
        assert digs == str(q) and E2 == E


def test_oracle_boundaries_of_fixed_notation():
    assert OJ.fmt(1, -14, 77) == "6.103515625e-05"           # E = -5: scientific
    assert OJ.fmt(1, -13, 77) == "0.0001220703125"            # E = -4: fixed
    assert OJ.fmt(10 ** 76, 0, 77) == "1" + "0" * 76          # E = p - 1: fixed
    assert OJ.fmt(10 ** 77, 0, 77) == "1e+77"                 # E = p: scientific
    assert OJ.fmt(0, 5, 77) == "0"


def test_oracle_poly_size_rule():
    s = OJ.eps_shift(77)
    one = (1 << 100, -100)
    assert OJ.poly_size([one, one, (0, 0)], 77) == 2
    assert OJ.poly_size([one, (1 << 100, -100 - s - 1)], 77) == 1          # below eps: dropped
    assert OJ.poly_size([one, (1 << 100, -100 - s + 1)], 77) == 2          # above eps: kept
    assert OJ.poly_size([(0, 0), (0, 0)], 77) == 0


@pytest.mark.parametrize("ci", range(len(JC.SPIN_CASES)))
def test_header_and_oracle_body_match_reference_files(ci):
    """complete files: the GPU writer's host header + the oracle's derivs body == the reference's write_spin"""
    g = golden("json_output.json")["spins"][ci]
    case = JC.SPIN_CASES[ci]
    opts, outputs, Sm, vals = JC.spin_case(case)
    pp = case[4]
    p = JO.digits10(opts.precision)
    for jo, tj in enumerate(opts.two_js_internal):
        structs = [(len(JC.so3(pp[k][0], opts.two_j12, tj)), len(JC.so3(pp[k][1], opts.two_j43, tj))) for k in range(2)]
        coord_rows = []
        for c in [c for c in JO.COORD_ORDER if c in opts.coordinates]:
            by_n = {}
            for oi, (n, _) in enumerate(outputs[c]):
                by_n.setdefault(n, []).append(oi)
            rows_idx = [by_n[n] for n in sorted(by_n)]

            def rows(k, s):
                return [[vals[c][jo][k][s][oi] for oi in row] for row in rows_idx]
            coord_rows.append([[[rows(k, a * Sm + b) for b in range(structs[k][1])] for a in range(structs[k][0])]
                               for k in range(2)])
        text = JO.header(opts, tj, pp, p) + "  \"derivs\":\n  [\n" + OJ.derivs_body(structs, coord_rows, p) + "\n  ]\n}\n"
        assert text == g["files"][str(tj)]
