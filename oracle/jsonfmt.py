"""CPU restatement of blocks_3d's per-spin JSON text as the reference's writer produces it
(``blocksvibe/b3djson.py``), for exact binary numbers m 2^e.  Test infrastructure only: the product's
formatter is the CUDA kernel pair behind ``b3d_format_decimal`` / ``b3d_emit_derivs``.

Numbers: the production writer turns every MPF into an MPFR number at the MPF's own precision (exact) and
prints it with MPFR's correctly rounded ``%.{p}g`` minus a trailing ``.0`` (``b3djson.py:56-66, 69-80``):
p significant digits rounded to nearest with ties to even, trailing zeros removed, fixed notation for
decimal exponents -4 <= E < p, else ``d.ddde+XX`` (at least two exponent digits).  The mpmath writer
(``fmt_big``, ``b3djson.py:32-53``) prints the same string except when the dropped digits are exactly one half
(it rounds those up); the golden fixtures come from it and hold no such ties.

Polynomials: blocks_3d drops negligible top coefficients (``b3djson.py:160-166``): scanning from the top
degree down, the kept size becomes d + 1 whenever |c_d| eps exceeds the largest magnitude above d, with
eps = 2^-(1 + int(0.9 log2(10) p)) (``b3djson.py:176-179``); an all-zero polynomial prints as ``"0"``.
"""
import math


def digits10(precision):
    """blocks_3d's output digits for an input precision in bits (``b3djson.py:20-23``)"""
    return ((precision - 1) // 64 + 1) * 64 * 301 // 1000


def eps_shift(p):
    """eps = 2^-eps_shift(p) (``b3djson.py:176-179``)"""
    return 1 + int(0.9 * math.log2(10) * p)


def decimal_digits(v, e, p):
    """|v| 2^e (v a nonzero int) -> (digit string of exactly p digits, decimal exponent E) with
    |v| 2^e ~= 0.d1d2...dp 10^(E+1), rounded to nearest, ties to even"""
    a = abs(v)
    num, den = (a << e, 1) if e >= 0 else (a, 1 << -e)
    E = len(str(num // den)) - 1 if num >= den else -len(str(den // num)) - 1
    while True:                                   # exact E with 10^E <= a 2^e < 10^(E+1)
        lo = (num * 10 ** -E, den) if E < 0 else (num, den * 10 ** E)
        if lo[0] < lo[1]:
            E -= 1
            continue
        hi = (num * 10 ** (-E - 1), den) if E + 1 < 0 else (num, den * 10 ** (E + 1))
        if hi[0] >= hi[1]:
            E += 1
            continue
        break
    k = p - 1 - E
    n2, d2 = (num * 10 ** k, den) if k >= 0 else (num, den * 10 ** -k)
    q, r = divmod(n2, d2)
    if 2 * r > d2 or (2 * r == d2 and q % 2):
        q += 1
    if q == 10 ** p:
        q //= 10
        E += 1
    return str(q), E


def fmt(v, e, p):
    """the printed form of v 2^e (v int, e int) at p significant digits"""
    if v == 0:
        return "0"
    digs, E = decimal_digits(v, e, p)
    digs = digs.rstrip("0") or "0"
    if E < -4 or E >= p:
        s = digs[0] + ("." + digs[1:] if len(digs) > 1 else "")
        s += "e" + ("-" if E < 0 else "+") + f"{abs(E):02d}"
    elif E >= 0:
        s = digs[:E + 1] + "." + digs[E + 1:] if len(digs) > E + 1 else digs + "0" * (E + 1 - len(digs))
    else:
        s = "0." + "0" * (-1 - E) + digs
    return ("-" if v < 0 else "") + s


def poly_size(poly, p):
    """kept size of one polynomial given as [(v, e), ...] (``b3djson.py:160-166``); 0 when all are zero"""
    if all(v == 0 for v, _ in poly):
        return 0
    s = eps_shift(p)
    size, mx = len(poly), (0, 0)                   # mx as an exact (numerator, power of two) pair
    for d in range(len(poly) - 1, -1, -1):
        v, e = poly[d]
        c = (abs(v), e)
        if _less(mx, (c[0], c[1] - s)):
            size = d + 1
        if _less(mx, c):
            mx = c
    return size


def _less(x, y):
    """x[0] 2^x[1] < y[0] 2^y[1] for nonnegative ints"""
    (a, ea), (b, eb) = x, y
    if a == 0 or b == 0:
        return a == 0 and b != 0
    m = min(ea, eb)
    return (a << (ea - m)) < (b << (eb - m))


def poly_text(poly, p):
    """one polynomial's lines inside its brackets (``b3djson.py:155-167``)"""
    size = poly_size(poly, p)
    if size == 0:
        return "\"0\""
    return ",\n".join(f"\"{fmt(v, e, p)}\"" for v, e in poly[:size])


def derivs_text(rows, p):
    """``b3djson.derivs_text`` (``b3djson.py:150-174``): rows[deriv_0][deriv_1] = polynomial"""
    out = ["          [\n"]
    for d0, row in enumerate(rows):
        out.append("            [\n")
        for d1, poly in enumerate(row):
            out.append("              [\n" + poly_text(poly, p) + "\n              ]")
            if d1 + 1 != len(row):
                out.append(",\n")
        out.append("\n            ]")
        if d0 + 1 != len(rows):
            out.append(",\n")
    out.append("\n          ]")
    return "".join(out)


def derivs_body(structs, coord_rows, p):
    """the ``"derivs"`` array of ``b3djson.write_spin`` (``b3djson.py:181-198``), without its opening
    ``  "derivs":\\n  [\\n`` and closing ``\\n  ]\\n}\\n``"""
    out = []
    for k in range(2):
        out.append("    [\n")
        nl, nr = structs[k]
        for a in range(nl):
            out.append("      [\n")
            for b in range(nr):
                out.append("        [\n")
                out.append(",\n".join(derivs_text(c[k][a][b], p) for c in coord_rows))
                out.append("\n        ]")
                if b + 1 != nr:
                    out.append(",\n")
            out.append("\n      ]")
            if a + 1 != nl:
                out.append(",\n")
        out.append("\n    ]")
        if k + 1 != 2:
            out.append(",\n")
    return "".join(out)
