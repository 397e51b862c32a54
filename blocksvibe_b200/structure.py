"""Pole and spin bookkeeping of blocks_3d's radial recursion (Erramilli et al., arXiv:2011.01959).

Spins are doubled integers (``tj = 2 j``), as in blocks_3d.  A pole is a pair ``(kind, k)`` with
``kind`` 0..3 for blocks_3d's pole types I..IV and ``k >= 1``.  The formulas are blocks_3d's
(Pole.hxx, Pole_Types.cxx, two_j_values.cxx, so3_tensor_parity.cxx, fill_residues.cxx) as restated
by the reference in ``blocksvibe/structure.py:16-127``; the conventions (pole order within a block,
type numbering) must be identical because slot layouts and key orders derive from them.

Scalar helpers work on Python ints; the ``*_v`` helpers work elementwise on numpy int64 arrays and
are what the vectorised plan builder uses.
"""
from fractions import Fraction
from functools import lru_cache

import numpy as np

KIND_I, KIND_II, KIND_III, KIND_IV = 0, 1, 2, 3


def is_boson(tj):
    return tj % 2 == 0


def kind_count(kind, tj, tj12, tj43, order):
    """number of poles of one kind in a block of spin tj truncated at ``order``
    (reference ``structure.py:16-24``)"""
    half = tj // 2
    narrow = min(half, tj12 // 2, tj43 // 2)
    if kind == KIND_I:
        n = order
    elif kind == KIND_II:
        n = min(half, order)
    elif kind == KIND_III:
        n = order // 2 if is_boson(tj) else min(narrow, order // 2)
    else:
        n = min(narrow, (order + 1) // 2) if is_boson(tj) else (order + 1) // 2
    return max(n, 0)


@lru_cache(maxsize=None)
def block_poles(tj, tj12, tj43, order):
    """poles of a block in blocks_3d's order: kind-major, k = 1, 2, ... (reference ``structure.py:28``)"""
    out = []
    for kind in range(4):
        out.extend((kind, k) for k in range(1, kind_count(kind, tj, tj12, tj43, order) + 1))
    return tuple(out)


def pole_index(tj, tj12, tj43, order, pole):
    """position of ``pole`` in ``block_poles(tj, tj12, tj43, order)`` (reference ``structure.py:32``)"""
    kind, k = pole
    return sum(kind_count(u, tj, tj12, tj43, order) for u in range(kind)) + k - 1


def level_shift(pole):
    """recursion-level offset of a pole (its order in r) (reference ``structure.py:37``)"""
    kind, k = pole
    if kind in (KIND_I, KIND_II):
        return k
    return 2 * k if kind == KIND_III else 2 * k - 1


def child_spin(pole, tj):
    """doubled spin of the block a pole's residue is proportional to (reference ``structure.py:42``)"""
    kind, k = pole
    if kind == KIND_I:
        return tj + 2 * k
    if kind == KIND_II:
        return tj - 2 * k
    return tj


def twice_position(pole, tj):
    """2 x the pole's position in Delta (reference ``structure.py:47-50``)"""
    kind, k = pole
    if kind == KIND_I:
        return 2 - tj - 2 * k
    if kind == KIND_II:
        return 4 + tj - 2 * k
    if kind == KIND_III:
        return 3 - 2 * k
    return 4 - 2 * k


def pole_parity(pole):
    return 1 if pole[0] == KIND_IV else 0


def residue_prefactor(pole, tj):
    """the exact rational Q(pole, tj) of fill_residues / Q.hxx (reference ``structure.py:56-64``)"""
    kind, k = pole
    scale = Fraction(4) ** level_shift(pole)
    if kind in (KIND_I, KIND_II):
        return -scale
    if kind == KIND_III:
        return -scale * Fraction(k * (1 + tj - 2 * k), 1 + tj + 2 * k)
    return scale * Fraction((2 + tj - 2 * k) * (2 * k - 1), 2 * tj + 4 * k)


def level_spins(m, order, tj12, tj_max):
    """doubled spins carried at recursion level m (reference ``structure.py:67``)"""
    return list(range(tj12 % 2, tj_max + 2 * (order - m - 1) + 1, 2))


@lru_cache(maxsize=None)
def so3_structures(pseudo_parity, tj1, tj2):
    """doubled spins of the SO(3) structures allowed by a pseudo-parity (reference ``structure.py:72``)"""
    return tuple(c for c in range(abs(tj1 - tj2), tj1 + tj2 + 1, 2)
                 if (tj1 + tj2 - c - 2 * pseudo_parity) % 4 == 0)


def spin_excess(tj, tj_max):
    """levels a spin above tj_max loses from its pole order (reference ``structure.py:77``)"""
    return (tj - tj_max) // 2 if tj > tj_max else 0


# ---------------------------------------------------------------- elementwise numpy versions

def _i64(*xs):
    return np.broadcast_arrays(*[np.asarray(x, dtype=np.int64) for x in xs])


def kind_counts_v(tj, tj12, tj43, order):
    """(4, *shape) int64 counts of the four pole kinds (reference ``structure.py:90-98``)"""
    tj, order = _i64(tj, order)
    half = tj // 2
    narrow = np.minimum(half, min(tj12 // 2, tj43 // 2))
    boson = tj % 2 == 0
    c = np.stack([order,
                  np.minimum(half, order),
                  np.where(boson, order // 2, np.minimum(narrow, order // 2)),
                  np.where(boson, np.minimum(narrow, (order + 1) // 2), (order + 1) // 2)])
    return np.maximum(c, 0)


def pole_at_v(tj, tj12, tj43, order, idx):
    """(kind, k) of the idx-th pole of each block (reference ``structure.py:101-107``)"""
    tj, order, idx = _i64(tj, order, idx)
    ends = np.cumsum(kind_counts_v(tj, tj12, tj43, order), axis=0)
    kind = (idx >= ends[0]).astype(np.int64) + (idx >= ends[1]) + (idx >= ends[2])
    begin = np.where(kind == 0, 0, np.take_along_axis(ends, np.maximum(kind - 1, 0)[None], 0)[0])
    return kind, idx - begin + 1


def pole_index_v(tj, tj12, tj43, order, kind, k):
    """position of (kind, k) within its block (reference ``structure.py:110-114``)"""
    tj, order, kind, k = _i64(tj, order, kind, k)
    ends = np.cumsum(kind_counts_v(tj, tj12, tj43, order), axis=0)
    begin = np.where(kind == 0, 0, np.take_along_axis(ends, np.maximum(kind - 1, 0)[None], 0)[0])
    return begin + k - 1


def level_shift_v(kind, k):
    return np.where(kind < 2, k, np.where(kind == 2, 2 * k, 2 * k - 1))


def child_spin_v(kind, k, tj):
    return np.where(kind == 0, tj + 2 * k, np.where(kind == 1, tj - 2 * k, tj))


def twice_position_v(kind, k, tj):
    return np.choose(kind, [2 - tj - 2 * k, 4 + tj - 2 * k, 3 - 2 * k, 4 - 2 * k])


def spin_excess_v(tj, tj_max):
    return np.where(tj > tj_max, (tj - tj_max) // 2, 0)
