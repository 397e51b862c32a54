"""Writes tests/golden/json_output.json by running the reference's JSON writer (BlocksviBe's
blocksvibe/b3djson.py, read from REFERENCE below) on the seeded values of json_cases.py:

  numbers  b3djson.fmt_big of exact values v 2^e at blocks_3d's digit counts (L = 10, 34, 42)
  spins    complete per-spin files of b3djson.write_spin (mpmath path: fmt_big numbers, the same truncation
           of negligible top coefficients), with the polynomials grouped per deriv_0 as cli._write_one
           groups them (cli.py:471-498)

b3djson imports gmpy2 (absent here) for its MPFR path only; an empty stand-in module is registered.  The
MPFR path prints the same strings except for values exactly halfway between two p-digit decimals, which
these seeded values do not contain.

    python tests/golden/make_json_golden.py REFERENCE
"""
import json
import os
import sys
import tempfile
import types

HERE = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) != 2:
    sys.exit(__doc__)
REFERENCE = sys.argv[1]
sys.path.insert(0, REFERENCE)
sys.path.insert(0, HERE)
sys.modules.setdefault("gmpy2", types.ModuleType("gmpy2"))

import mpmath as mp                                  # noqa: E402
from mpmath import libmp                             # noqa: E402
from blocksvibe import b3djson as BJ                 # noqa: E402
import json_cases as JC                              # noqa: E402


def exact(v, e):
    return mp.mp.make_mpf(libmp.from_man_exp(v, e))


def make_numbers():
    out = []
    for L, count, seed in JC.NUMBER_CASES:
        p = BJ.digits10(32 * (L - 2))
        vals = JC.random_numbers(L, count, seed)
        out.append({"L": L, "count": count, "seed": seed, "p": p,
                    "text": [BJ.fmt_big(exact(v, e), p) for v, e in vals]})
    return out


def make_spins():
    out = []
    for ci, case in enumerate(JC.SPIN_CASES):
        opts, outputs, Sm, vals = JC.spin_case(case)
        pp = case[4]
        files = {}
        for jo, tj in enumerate(opts.two_js_internal):
            structs = [(len(JC.so3(pp[k][0], opts.two_j12, tj)), len(JC.so3(pp[k][1], opts.two_j43, tj)))
                       for k in range(2)]
            coord_rows = []
            for c in [c for c in BJ.COORD_ORDER if c in opts.coordinates]:
                by_n = {}
                for oi, (n, _) in enumerate(outputs[c]):
                    by_n.setdefault(n, []).append(oi)
                rows_idx = [by_n[n] for n in sorted(by_n)]

                def rows(k, s):
                    return [[[exact(v, e) for v, e in vals[c][jo][k][s][oi]] for oi in row] for row in rows_idx]
                coord_rows.append([[[rows(k, a * Sm + b) for b in range(structs[k][1])] for a in range(structs[k][0])]
                                   for k in range(2)])
            with tempfile.TemporaryDirectory() as d:
                path = os.path.join(d, "spin.json")
                BJ.write_spin(path, opts, tj, pp, structs, coord_rows, gmp=False)
                with open(path) as f:
                    files[str(tj)] = f.read()
        out.append({"case": ci, "files": files})
    return out


if __name__ == "__main__":
    res = {"numbers": make_numbers(), "spins": make_spins()}
    path = os.path.join(HERE, "json_output.json")
    with open(path, "w") as f:
        json.dump(res, f)
    print(path, os.path.getsize(path))
