"""Oracle bookkeeping: poles and spins of blocks_3d's recursion, written as plain loops over Python ints.
Follows the reference's blocksvibe/structure.py:16-84 (a 1:1 port of blocks_3d's Pole.hxx,
Pole_Types.cxx, two_j_values.cxx, so3_tensor_parity.cxx).  Test infrastructure only."""
from fractions import Fraction


def pole_list(tj, tj12, tj43, order):
    """[(kind, k)] kind 0..3 = types I..IV, kind-major (structure.py:16-29)"""
    boson = tj % 2 == 0
    small = min(tj // 2, tj12 // 2, tj43 // 2)
    counts = [order,
              min(tj // 2, order),
              order // 2 if boson else min(small, order // 2),
              min(small, (order + 1) // 2) if boson else (order + 1) // 2]
    return [(kind, k) for kind in range(4) for k in range(1, max(counts[kind], 0) + 1)]


def shift(pole):
    kind, k = pole
    return (k, k, 2 * k, 2 * k - 1)[kind]


def child(pole, tj):
    kind, k = pole
    return (tj + 2 * k, tj - 2 * k, tj, tj)[kind]


def twice_pos(pole, tj):
    kind, k = pole
    return (2 - tj - 2 * k, 4 + tj - 2 * k, 3 - 2 * k, 4 - 2 * k)[kind]


def q_value(pole, tj):
    """Q.hxx (structure.py:56-64)"""
    kind, k = pole
    four = Fraction(4) ** shift(pole)
    if kind < 2:
        return -four
    if kind == 2:
        return -four * Fraction(k * (1 + tj - 2 * k), 1 + tj + 2 * k)
    return four * Fraction((2 + tj - 2 * k) * (2 * k - 1), 2 * tj + 4 * k)


def spins(m, order, tj12, tj_max):
    return list(range(tj12 % 2, tj_max + 2 * (order - m - 1) + 1, 2))


def so3(pp, tj1, tj2):
    return [c for c in range(abs(tj1 - tj2), tj1 + tj2 + 1, 2) if ((tj1 + tj2 - c) - 2 * pp) % 4 == 0]


def excess(tj, tj_max):
    return (tj - tj_max) // 2 if tj > tj_max else 0
