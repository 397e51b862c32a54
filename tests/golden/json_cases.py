"""Seeded inputs of the JSON-output fixtures, shared by make_json_golden.py (which runs the reference's writer
on them) and the tests (which run the oracle and the GPU writer on the same values).  Pure Python: the
same seed gives the same numbers everywhere.

Numbers are exact binary values v 2^e with v an NB = 32 L - 2 bit signed integer, as the drop-in's MPF
arrays hold them."""
import random
from types import SimpleNamespace

NUMBER_CASES = [  # (L, count, seed)
    (10, 120, 101), (34, 40, 134), (42, 40, 142)]

# exact values with short decimal forms (integers, dyadic fractions) and format boundaries
SPECIAL = [(1, 0), (-1, 0), (1, -1), (3, -2), (1, -10), (5, -14), (-7, -20), (1, 40), (10 ** 20, 0),
           (999999, -20), (1, -13), (1, -14), (123456789, -30)]

SPIN_CASES = [  # (precision, coords, Lambda, sign, pp, tj12, tj43, two_js_internal, Dmax, seed)
    (256, ("xt",), 3, 1, ((0, 0), (1, 1)), 2, 2, [0, 2], 3, 201),
    (256, ("xt", "xt_radial"), 3, -1, ((0, 1), (1, 0)), 2, 2, [2, 4], 3, 202),
    (512, ("xt_radial",), 4, 1, ((0, 0), (1, 1)), 1, 1, [1, 3], 4, 203),
]


def nb_bits(L):
    return 32 * L - 2


def random_numbers(L, count, seed):
    """count values (v, e): normalised NB-bit mantissas, decimal exponents from about 10^-(2p) to 10^(p+40),
    plus SPECIAL"""
    rng = random.Random(seed)
    NB = nb_bits(L)
    p = 32 * (L - 2) * 301 // 1000
    out = list(SPECIAL)
    for _ in range(count):
        v = rng.getrandbits(NB - 1) | (1 << (NB - 1))
        if rng.random() < 0.5:
            v = -v
        E10 = rng.choice([rng.randint(-2 * p, p + 40), rng.randint(-6, 6), rng.randint(p - 3, p + 1)])
        out.append((v, int(E10 * 3.3219280948873626) - NB + rng.randint(-2, 2)))
    return out


def xt_outputs(O, parity):
    return [(n, b) for n in range(O - parity + 1) for b in range((O - n - parity) // 2 + 1)]


def radial_outputs(O, parity):
    return [(i, 0) for i in range(O - parity + 1)]


def so3(pp, tj1, tj2):
    return [c for c in range(abs(tj1 - tj2), tj1 + tj2 + 1, 2) if (tj1 + tj2 - c - 2 * pp) % 4 == 0]


def spin_case(case):
    """(options namespace, outputs {coord: list}, Smax, values {coord: nested list [jo][k][s][o][d] of (v, e)})"""
    prec, coords, Lam, sign, pp, tj12, tj43, tjs_int, Dmax, seed = case
    L = 2 * ((prec + 63) // 64) + 2
    NB = nb_bits(L)
    rng = random.Random(seed)
    parity = (1 - sign) // 2
    outputs = {}
    for c in coords:
        outputs[c] = xt_outputs(Lam, parity) if c == "xt" else radial_outputs(Lam - parity, parity)
    Sm = max(len(so3(pp[k][i], (tj12, tj43)[i], tj)) for tj in tjs_int for k in range(2) for i in range(2))
    opts = SimpleNamespace(two_js=(2, 2, 2, 2), two_j12=tj12, two_j43=tj43, delta_12="0.25", delta_43="-0.5",
                           delta_1_plus_2="2.3", q4=(1, 2, 1, 0), sign=sign, order=2 * Lam + 6, Lambda=Lam,
                           kept_pole_order=Lam + 3, coordinates=coords, precision=prec,
                           two_js_internal=list(tjs_int), out_template="out/spin_{}.json",
                           argv=["--precision", str(prec), "-o", "out/spin_{}.json"])
    vals = {}
    for c in coords:
        per = []
        for _ in tjs_int:
            ks = []
            for k in range(2):
                ss = []
                for s in range(Sm * Sm):
                    os_ = []
                    for o in range(len(outputs[c])):
                        poly = []
                        kind = rng.random()
                        for d in range(Dmax):
                            if kind < 0.1 or (kind < 0.3 and d == Dmax - 1):
                                poly.append((0, 0))                     # all-zero polynomial / zero top
                                continue
                            v = rng.getrandbits(NB - 1) | (1 << (NB - 1))
                            if rng.random() < 0.5:
                                v = -v
                            E10 = rng.randint(-30, 30)
                            if 0.3 <= kind < 0.45 and d == Dmax - 1:
                                E10 -= 400                              # negligible top coefficient
                            poly.append((v, int(E10 * 3.32) - NB))
                        os_.append(poly)
                    ss.append(os_)
                ks.append(ss)
            per.append(ks)
        vals[c] = per
    return opts, outputs, Sm, vals
