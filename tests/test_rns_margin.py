"""The CRT quotient of the residue GEMM on the host (CPU only): both reconstruction kernels form
x' = sum_j y_j M / p_j = P + q M exactly and take q = round(x' / M) in 64-bit integers from two words of x'
(crt_quotient in csrc/rns.cuh, restated as rns.crt_quotient), which is exact while |P| stays inside M / 8.
Checked for every compiled limb count: the prime set's M against the largest product the kernels can meet
(K = 4096 terms of two NB-bit magnitudes), the bounds the integer estimate needs (x' < 2^(32 msw + 63),
M / 2^(32 msw) >= 2^23), and the quotient on adversarial products: the largest positive and negative ones,
zero, +-1, and products whose x' / M lies as close to a half-integer as the margin allows."""
import random
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
def test_integer_quotient_on_adversarial_products(L):
    npr, ml, ps, M, inv = _setup(L)
    NB = 32 * L - 2
    msw, mtop = rns.crt_quotient_words(M)
    assert mtop >= 1 << 23 and npr * M < 1 << (32 * msw + 63) and msw + 1 < ml + 1
    pmax = KMAX * ((1 << NB) - 1) ** 2
    rng = random.Random(L)
    cases = [pmax, -pmax, 0, 1, -1, (1 << (2 * NB)) - 1, -(1 << (2 * NB))]
    cases += [rng.randrange(-pmax, pmax + 1) for _ in range(40)]
    cases += [pmax - rng.randrange(1 << 40) for _ in range(10)] + [-pmax + rng.randrange(1 << 40) for _ in range(10)]
    for P in cases:
        ys = [(P % p) * i % p for p, i in zip(ps, inv)]
        xp = sum(y * (M // p) for y, p in zip(ys, ps))
        assert xp % M == P % M and 0 <= xp < npr * M
        q = rns.crt_quotient(xp, msw, mtop)
        assert xp - q * M == P, (L, P)


def test_integer_quotient_is_round_to_nearest_across_its_range():
    """the estimate against exact rounding for x' / M anywhere within 1/8 of an integer 0 .. np"""
    npr, ml, ps, M, _ = _setup(34)
    msw, mtop = rns.crt_quotient_words(M)
    rng = random.Random(5)
    for _ in range(2000):
        q = rng.randrange(0, npr + 1)
        off = rng.randrange(-(M // 8) + 1, M // 8)
        xp = q * M + off
        if xp < 0:
            continue
        assert rns.crt_quotient(xp, msw, mtop) == q
