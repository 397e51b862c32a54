"""Seeded inputs of the full-size chain fixtures (make_chain_golden.py writes the oracle's results for them,
tests/test_gpu_fullsize.py runs the GPU chain on them).

Every input number is a dyadic rational drawn from a hash of (case seed, what it is, its key), so the oracle
(mpmath, dict of lazily built entries) and the GPU test (tables in the plan's key order) see the same exact
values without storing them:
  M entries    k 2^-198 with k a signed 200-bit integer (|M| < 2)
  h_inf        k 2^-199 with k a signed 200-bit integer (|h| < 1)

Cases:
  cfg2_n0      the bench's default configuration: j = (2,2,2,2), 2j12 = 2j43 = 8, spins 0-44 (doubled), order
               40, Lambda 11, kept pole order 20 (pole shifting on), 1024 bits (L = 34); lambda order n = 0
               (R = 11): residues of sampled (parity, level, spin, pole) blocks and numerators of sampled
               (spin, parity, structure) blocks
  cfg5_radial  the largest configuration's shape restricted to output spins 0-4: 2j12 = 2j43 = 8, order 80,
               Lambda 27, kept pole order 40 (pole shifting on), 1280 bits (L = 42), xt_radial, Delta_1+2 = 6;
               lambda order n = parity = 0 (R = 27): residues of sampled blocks and the xt_radial outputs of
               sampled (spin, parity, structure) blocks
"""
import hashlib

CASES = {
    "cfg2_n0": dict(tj12=8, tj43=8, tjmax=44, order=40, Lam=11, n=0, kept=20, precision=1024, L=34,
                    pp=((0, 0), (1, 1)), seed=2002, res_blocks=80, num_blocks=6, coord=None, d12="6"),
    "cfg5_radial": dict(tj12=8, tj43=8, tjmax=4, order=80, Lam=27, n=0, kept=40, precision=1280, L=42,
                        pp=((0, 0), (1, 1)), seed=5005, res_blocks=40, num_blocks=2, coord="xt_radial", d12="6"),
}


def _signed(seed, tag, key, bits=200):
    h = hashlib.blake2b(f"{seed}|{tag}|{key!r}".encode(), digest_size=(bits + 8) // 8 + 1).digest()
    k = int.from_bytes(h, "little") & ((1 << (bits + 1)) - 1)
    return k - (1 << bits)


def m_entry(seed, key, a, b):
    """(integer, exponent) of M[key][a][b]"""
    return _signed(seed, "M", (key, a, b)), -198


def h_entry(seed, src, m, jh, a, b):
    """(integer, exponent) of h_inf[(src, m, jh, a, b)]"""
    return _signed(seed, "h", (src, m, jh, a, b)), -199


def so3(pp, tj1, tj2):
    return [c for c in range(abs(tj1 - tj2), tj1 + tj2 + 1, 2) if ((tj1 + tj2 - c) - 2 * pp) % 4 == 0]


def m_shape(key):
    """(rows, columns) of blocks_3d's M matrix of a key (pole, side, tjNN, pseudo-parity, tj)"""
    (kind, k), _, tjnn, ppq, tj = key
    child = (tj + 2 * k, tj - 2 * k, tj, tj)[kind]
    return len(so3((ppq + (1 if kind == 3 else 0)) % 2, tjnn, tj)), len(so3(ppq, tjnn, child))


def encode(vals, bits):
    """a block of mpmath numbers as (E, [hex]) with v = int 2^(E - bits), E the top exponent of the block"""
    import mpmath as mp
    E = None
    for v in vals:
        if v:
            e = int(mp.frexp(v)[1])
            E = e if E is None else max(E, e)
    if E is None:
        return 0, ["0"] * len(vals)
    return E, [format(int(mp.nint(mp.ldexp(v, bits - E))), "x") for v in vals]


def decode(E, hexes, bits):
    import mpmath as mp
    return [mp.ldexp(mp.mpf(int(h, 16)), E - bits) for h in hexes]
