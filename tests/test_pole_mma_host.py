"""The rounding of the tensor-core pole step, restated on the host (CPU only).

k_pole_mma (csrc/pole_mma.cuh) rounds each exact sum in two parts: one header thread per column decides the
rounding from the two's complement limb column (pm_head: sign, lowest nonzero limb z, bit length, shift
s = bl - NB, half bit c0, the limbs kc the rounding carry reaches, the lowest nonzero rounded limb kz, or the
renormalisation when the carry reaches 2^NB), and every output limb is then formed on its own (pm_limb /
pm_limbs).  This file restates those formulas limb for limb and checks them against the rounding rule of the
package (round_mag: NB bits, half away from zero on the magnitude) on magnitudes chosen to reach the rare
branches: carries through runs of all-ones limbs, the renormalisation, rounded values with zero low limbs
(the two's complement negation starting above them), and negative sums.  It also restates the carry chains in
segments of eight limbs and the header's join of their carries, against exact sums for every tile geometry, and
the operand layout: the Hankel windows and reversed column digits read through the MMAs' descriptors give the
exact dot products as byte positions."""
import random

import pytest

M32 = (1 << 32) - 1


def limbs(v, n):
    return [(v >> (32 * k)) & M32 for k in range(n)]


def fsr(lo, hi, f):
    return ((lo | (hi << 32)) >> f) & M32


class Col:
    """PmCol: the magnitude view of a two's complement column of NW limbs"""

    def __init__(self, col, NW):
        self.col, self.NW = col, NW
        self.neg = (col[NW - 1] >> 31) != 0
        self.z = 0
        if self.neg:
            while self.z < NW - 1 and col[self.z] == 0:
                self.z += 1

    def conv(self, i, v):
        if not self.neg:
            return v
        return (~v) & M32 if i > self.z else ((-v) & M32 if i == self.z else 0)

    def __call__(self, i):
        return 0 if i < 0 or i >= self.NW else self.conv(i, self.col[i])

    def bitlen(self):
        for i in range(self.NW - 1, -1, -1):
            m = self(i)
            if m:
                return 32 * i + m.bit_length()
        return 0


def head(m, bl, L):
    """pm_head: (mode, s, Q, F, c0, kc, kz); mode 'limbs', 'renorm' or 'done' (s <= 0)"""
    NB = 32 * L - 2
    s = bl - NB
    if s <= 0:
        return "done", s, 0, 0, 0, -1, 0
    Q, F = s >> 5, s & 31
    c0 = (m((s - 1) >> 5) >> ((s - 1) & 31)) & 1
    x = lambda k: fsr(m(Q + k), m(Q + k + 1), F)                 # noqa: E731
    if c0:
        k, xk = 0, x(0)
        while xk == M32 and k < L - 1:
            k += 1
            xk = x(k)
        mode = "renorm" if k == L - 1 and xk + 1 == 1 << (NB - 32 * (L - 1)) else "limbs"
        return mode, s, Q, F, c0, k, k
    k = 0
    while k < L - 1 and x(k) == 0:
        k += 1
    return "limbs", s, Q, F, c0, -1, k


def limb(h, m, k, L):
    """pm_limb: limb k of the stored two's complement result"""
    NB = 32 * L - 2
    mode, s, Q, F, c0, kc, kz = h
    if mode == "renorm":
        r = 1 << (NB - 1 - 32 * (L - 1)) if k == L - 1 else 0
        return ((-r) & M32 if k == L - 1 else 0) if m.neg else r
    r = (fsr(m(Q + k), m(Q + k + 1), F) + (1 if k <= kc else 0)) & M32
    if not m.neg:
        return r
    return 0 if k < kz else ((-r) & M32 if k == kz else (~r) & M32)


def kernel_round(v, L):
    """the kernel's rounding of the exact sum v: (stored value, shift) or None for zero"""
    NW = 2 * L + 2
    m = Col(limbs(v % (1 << (32 * NW)), NW), NW)
    bl = m.bitlen()
    if bl == 0:
        return None
    h = head(m, bl, L)
    assert h[0] != "done"
    out = [limb(h, m, k, L) for k in range(L)]
    val = sum(w << (32 * k) for k, w in enumerate(out))
    if val >> (32 * L - 1):
        val -= 1 << (32 * L)
    return val, h[1] + (1 if h[0] == "renorm" else 0)


def expected_round(v, L):
    """round_mag: |v| to NB bits, half away from zero; the sign applied after"""
    NB = 32 * L - 2
    a = abs(v)
    if a == 0:
        return None
    s = a.bit_length() - NB
    t = a >> (s - 1)
    r = (t >> 1) + (t & 1)
    if r >> NB:
        r >>= 1
        s += 1
    return (-r if v < 0 else r), s


def adversarial(L, rng):
    NB = 32 * L - 2
    top = 2 * NB + 2                                              # bit length of a five-term sum at most
    out = []
    for _ in range(60):
        bl = rng.randrange(NB + 1, top + 1)
        s = bl - NB
        kind = rng.randrange(6)
        if kind == 0:                                             # all ones down to the half bit: renormalises
            a = ((1 << NB) - 1) << s | (1 << (s - 1)) | rng.getrandbits(max(s - 1, 0))
        elif kind == 1:                                           # a run of all-ones limbs above the half bit
            run = rng.randrange(1, L)
            a = (rng.getrandbits(NB - 32 * run) | 1 << (NB - 32 * run - 1)) << (32 * run + s)
            a |= ((1 << (32 * run)) - 1) << s | 1 << (s - 1) | rng.getrandbits(max(s - 1, 0))
        elif kind == 2:                                           # zero low limbs in the rounded value
            zl = rng.randrange(1, L)
            a = (rng.getrandbits(NB - 32 * zl) | 1 << (NB - 32 * zl - 1)) << (32 * zl + s)
            a |= rng.getrandbits(max(s - 1, 0))                   # half bit clear
        elif kind == 3:                                           # exactly at a midpoint
            a = (rng.getrandbits(NB - 1) | 1 << (NB - 1)) << s | 1 << (s - 1)
        elif kind == 4:                                           # just below a midpoint
            a = (rng.getrandbits(NB - 1) | 1 << (NB - 1)) << s | ((1 << (s - 1)) - 1)
        else:
            a = rng.getrandbits(bl) | 1 << (bl - 1)
        out.append(a)
        out.append(-a)
    return out


@pytest.mark.parametrize("L", [10, 18, 26, 34, 42, 46])
def test_header_and_limb_formulas_round_like_round_mag(L):
    rng = random.Random(L)
    for v in adversarial(L, rng):
        assert kernel_round(v, L) == expected_round(v, L), (L, v)


def test_adversarial_cases_reach_every_branch():
    L = 34
    rng = random.Random(1)
    seen = set()
    for v in adversarial(L, rng):
        NW = 2 * L + 2
        m = Col(limbs(v % (1 << (32 * NW)), NW), NW)
        h = head(m, m.bitlen(), L)
        seen.add(h[0])
        if h[5] > 0:
            seen.add("carry run")
        if h[6] > 0 and m.neg:
            seen.add("negation above zero limbs")
    assert {"limbs", "renorm", "carry run", "negation above zero limbs"} <= seen


def chain_segments(V, NW, lo, nseg):
    """the carry-chain segments of k_pole_mma: words V[w] (signed, four positions each) chained in segments of
    eight from a zero carry into limbs lo + w; returns the limb column and each segment's carry out"""
    col = [0] * NW
    carr = []
    for sg in range(nseg):
        c = 0
        for q in range(8):
            k = lo + 8 * sg + q
            if k < NW:
                s = c + V[8 * sg + q]
                col[k] = s & M32
                c = s >> 32
        carr.append(c)
    return col, carr


def join_segments(col, carr, NW, lo, nseg):
    """the header's join: segment sg receives the carry out of segment sg - 1 (all at once), then what runs
    out of the top of a segment is passed on in order; the sign-extension limbs above the last segment"""
    col = col[:]
    e = []
    for sg in range(nseg):
        c = carr[sg - 1] if sg > 0 else 0
        k = lo + 8 * sg
        kend = min(k + 8, NW)
        while c != 0 and k < kend:
            v = col[k] + c
            col[k], c = v & M32, v >> 32
            k += 1
        e.append(c)
    x = 0
    for sg in range(1, nseg):
        x += e[sg - 1]
        k = lo + 8 * sg
        kend = min(k + 8, NW)
        while x != 0 and k < kend:
            v = col[k] + x
            col[k], x = v & M32, v >> 32
            k += 1
    C = carr[nseg - 1] + x + e[nseg - 1]
    for k in range(lo + 8 * nseg, NW):
        col[k], C = C & M32, C >> 32
    return col


@pytest.mark.parametrize("L,P0,MT", [(10, 0, 1), (18, 16, 1), (26, 80, 1), (30, 0, 2), (34, 16, 2), (42, 80, 2),
                                     (46, 112, 2)])
def test_segment_carry_join_gives_the_exact_sum(L, P0, MT):
    """every tile geometry of the kernel: the joined column equals the exact sum of the words (mod 2^(32 NW)),
    also when carries run through whole segments (words drawn from all-ones, zero and -1 runs)"""
    NW, lo, nseg = 2 * L + 2, P0 // 4, 4 * MT
    rng = random.Random(L)
    for it in range(400):
        V = [rng.randrange(-(1 << 48), 1 << 48) for _ in range(8 * nseg)]
        if it % 2:
            V = [rng.choice([M32, 0, -1, M32 - 1]) if rng.random() < 0.7 else v for v in V]
        for w in range(8 * nseg):                                 # words above the accumulator carry nothing
            if lo + w >= NW:
                V[w] = 0
        col, carr = chain_segments(V, NW, lo, nseg)
        got = join_segments(col, carr, NW, lo, nseg)
        exact = sum(v << (32 * (lo + w)) for w, v in enumerate(V)) % (1 << (32 * NW))
        assert got == limbs(exact, NW), (L, it)


def _geometry(L):
    NB, D = 32 * L - 2, 4 * L
    U = 32 * (-(-D // 32))

    def p0(mt):
        top = 8 * L - 1 - 128 * mt
        return 0 if top <= 0 else 16 * (-(-top // 16))
    MT = 1 if 8 * p0(1) + 17 <= NB - 160 else 2
    return U, MT, p0(MT)


def balanced_digits(v, L):
    """the bytes of v + 0x8080...80 (4 L bytes), each minus 128: v = sum_u d_u 256^u, d_u in [-128, 127]"""
    t = v + int("80" * (4 * L), 16)
    assert 0 <= t < 1 << (32 * L)
    return [((t >> (8 * u)) & 0xFF) - 128 for u in range(4 * L)]


def descriptor_matrix(buf, start, lbo, sbo, rows, kbytes):
    """the rows x kbytes int8 matrix a canonical no-swizzle K-major descriptor addresses: core matrices of 8 rows
    x 16 bytes, (row group g, K chunk q) at start + g sbo + q lbo, row r of a core matrix at + 16 r"""
    import numpy as np
    m = np.zeros((rows, kbytes), dtype=np.int64)
    for row in range(rows):
        for k in range(kbytes):
            m[row, k] = buf[start + (row // 8) * sbo + (k // 16) * lbo + (row % 8) * 16 + k % 16]
    return m


@pytest.mark.parametrize("L,S,ncols", [(10, 3, 16), (10, 2, 32), (26, 2, 16), (30, 2, 16), (34, 2, 16)])
def test_hankel_windows_and_reversed_digits_give_the_exact_sums(L, S, ncols):
    """one row of a task: the byte windows of the constant's digit strings (16 bytes per offset, descriptor
    LBO 256, SBO 128) against the reversed column digits (LBO 16 NC, SBO 128) give, through the MMAs' K steps
    and tiles, D[p, n] whose positions from P0 sum to the exact dot products (up to the dropped low part)"""
    import numpy as np
    U, MT, P0 = _geometry(L)
    NB = 32 * L - 2
    rng = random.Random(L * 7 + S)
    c = [rng.randrange(-(1 << NB) + 1, 1 << NB) for _ in range(S)]                  # row i of the constant
    x = [[rng.randrange(-(1 << NB) + 1, 1 << NB) for _ in range(ncols)] for _ in range(S)]   # X[j][n]
    # the windows: padded digit string (U zero bytes first), window o (o < NWIN) = 16 bytes from byte P0 + 1 + o
    NWIN, FAM = 128 * MT + U - 16, 16 * (128 * MT + U - 16)
    hank = bytearray(S * FAM)
    for j in range(S):
        pad = [0] * U + [d & 0xFF for d in balanced_digits(c[j], L)] + [0] * (P0 + 128 * MT + U)
        for o in range(NWIN):
            hank[j * FAM + 16 * o: j * FAM + 16 * o + 16] = bytes(pad[P0 + 1 + o: P0 + 17 + o])
    hank = np.frombuffer(bytes(hank), dtype=np.int8)
    # the B operand: column n, K index j U + u' holds digit U - 1 - u' of x[j][n]
    bop = bytearray(S * U * ncols)
    for j in range(S):
        for n in range(ncols):
            d = balanced_digits(x[j][n], L) + [0] * (U - 4 * L)
            for up in range(U):
                kap = j * U + up
                bop[(kap // 16) * 16 * ncols + (n // 8) * 128 + (n % 8) * 16 + kap % 16] = d[U - 1 - up] & 0xFF
    bop = np.frombuffer(bytes(bop), dtype=np.int8)
    D = np.zeros((128 * MT, ncols), dtype=np.int64)
    for mt in range(MT):
        for j in range(S):
            for ks in range(U // 32):
                A = descriptor_matrix(hank, j * FAM + 2048 * mt + 512 * ks, 256, 128, 128, 32)
                B = descriptor_matrix(bop, (j * (U // 16) + 2 * ks) * 16 * ncols, 16 * ncols, 128, ncols, 32)
                D[128 * mt:128 * mt + 128] += A @ B.T
    assert np.abs(D).max() < 1 << 31
    for n in range(ncols):
        exact = sum(c[j] * x[j][n] for j in range(S))
        got = sum(int(D[p, n]) << (8 * (P0 + p)) for p in range(128 * MT))
        low = 0                                                         # positions below P0, exactly
        for pp in range(P0):
            for j in range(S):
                dc, dx = balanced_digits(c[j], L), balanced_digits(x[j][n], L)
                low += sum(dc[q] * dx[pp - q] for q in range(max(0, pp - 4 * L + 1), min(pp, 4 * L - 1) + 1)) << (8 * pp)
        assert got + low == exact, (L, n)
        assert abs(exact - got) < 1 << (8 * P0 + 17)                   # the dropped part's bound
