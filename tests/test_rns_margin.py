"""The CRT quotient of the residue GEMM on the host (CPU only): both reconstruction kernels estimate
q = round(x' / M) in double precision, x' = sum_j y_j M / p_j = P + q M, and are exact only while |P| stays
well inside M / 4.  Checked for every compiled limb count: the prime set's M against the largest product the
kernels can meet (K = 4096 terms of two NB-bit magnitudes), and both kernels' double-precision quotient
(k_rns_crt_mma: from the top four limbs of x' and of M; k_rns_crt: sum_j y_j (1 / p_j)) emulated in IEEE
doubles on adversarial products: the largest positive and negative ones, zero, +-1, and products whose x' / M
lies as close to a half-integer as the margin allows."""
import random
import struct
from math import prod

import pytest

from blocksvibe_b200 import rns

LIMBS = (6, 10, 14, 18, 22, 26, 30, 34, 38, 42, 46)
KMAX = 4096


def _setup(L):
    npr, ml = rns.layout(L)
    ps = rns.primes_below_2_31(npr)
    M = prod(ps)
    inv = [pow(M // p, -1, p) for p in ps]
    return npr, ml, ps, M, inv


def _limbs(x, n):
    return [(x >> (32 * c)) & 0xFFFFFFFF for c in range(n)]


def _quotient_mma(xp, M, ml):
    """k_rns_crt_mma: xt over limbs NX - 1 .. ML - 4 of x', mt over ML - 1 .. ML - 4 of M, llrint(xt / mt)"""
    NX = ml + 2
    x, m = _limbs(xp, NX), _limbs(M, ml)
    xt = 0.0
    for c in range(NX - 1, ml - 5, -1):
        xt = xt * 4294967296.0 + float(x[c])
    mt = 0.0
    for c in range(ml - 1, ml - 5, -1):
        mt = mt * 4294967296.0 + float(m[c])
    return round(xt / mt)                  # llrint in the default rounding mode: nearest, ties to even


def _quotient_cuda(ys, ps):
    """k_rns_crt: f = sum_j y_j * (1 / p_j) in double, llrint(f)"""
    f = 0.0
    for y, p in zip(ys, ps):
        rp = struct.unpack("d", struct.pack("d", 1.0 / p))[0]
        f += float(y) * rp
    return round(f)


@pytest.mark.parametrize("L", LIMBS)
def test_prime_set_covers_the_largest_product_with_margin(L):
    npr, ml, ps, M, _ = _setup(L)
    NB = 32 * L - 2
    pmax = KMAX * ((1 << NB) - 1) ** 2
    assert all(2 ** 30 < p < 2 ** 31 for p in ps) and len(set(ps)) == npr
    assert M > 4 * pmax
    assert M.bit_length() <= 32 * ml
    # |P| / M < 1/8: x' / M lies within 1/8 of an integer, 3/8 away from any half-integer
    assert 8 * pmax < M


@pytest.mark.parametrize("L", LIMBS)
def test_double_precision_quotients_on_adversarial_products(L):
    npr, ml, ps, M, inv = _setup(L)
    NB = 32 * L - 2
    pmax = KMAX * ((1 << NB) - 1) ** 2
    rng = random.Random(L)
    cases = [pmax, -pmax, 0, 1, -1, (1 << (2 * NB)) - 1, -(1 << (2 * NB))]
    cases += [rng.randrange(-pmax, pmax + 1) for _ in range(40)]
    cases += [pmax - rng.randrange(1 << 40) for _ in range(10)] + [-pmax + rng.randrange(1 << 40) for _ in range(10)]
    for P in cases:
        ys = [(P % p) * i % p for p, i in zip(ps, inv)]
        xp = sum(y * (M // p) for y, p in zip(ys, ps))
        assert xp % M == P % M and 0 <= xp < npr * M
        for q in (_quotient_mma(xp, M, ml), _quotient_cuda(ys, ps)):
            assert xp - q * M == P, (L, P)
