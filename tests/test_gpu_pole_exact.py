"""The pole step (b3d_pole_level on the CUDA cores, b3d_pole_level_mma on the tensor cores) on sums built to
cancel, against an exact restatement in Python integers.

Both forms first form the sums without their lowest part (limb columns on the CUDA cores, byte positions below
the first 128-lane tile on the tensor cores) and keep that rounding only where no value within the dropped
part rounds differently; elsewhere they redo the sum exactly.  Here the R and QL tables
have a negated column and H repeats rows with one bit flipped, so both stages meet exact zeros and
cancellations of every depth (the exact redo), next to ordinary sums (the first try).  Every result must
equal the exact sum of the aligned operands rounded once, half away from zero: the rule of every aligned
product of the package (mpf.gemm_aligned and the tensor-core residue GEMM give the same bits)."""
import random

import pytest
import torch

from blocksvibe_b200 import _lib, mpf

pytestmark = pytest.mark.gpu


def _align(vals, L):
    """sign-magnitude mantissas shifted to the largest exponent of the nonzero entries (truncated), and it"""
    nz = [e for v, e in vals if v != 0]
    if not nz:
        return [0] * len(vals), mpf.EZ
    E = max(nz)
    out = []
    for v, e in vals:
        if v == 0 or E - e >= 32 * L:
            out.append(0)
            continue
        a = abs(v) >> (E - e)
        out.append(-a if v < 0 else a)
    return out, E


def _dot(avals, bvals, L):
    A, Ea = _align(avals, L)
    B, Eb = _align(bvals, L)
    if Ea == mpf.EZ or Eb == mpf.EZ:
        return 0, mpf.EZ
    return mpf._round(sum(x * y for x, y in zip(A, B)), Ea + Eb, mpf.nbits(L))


def _case(L, S, B, T, seed):
    rng = random.Random(seed)
    NB = mpf.nbits(L)

    def rnd(spread=6):
        v = rng.getrandbits(NB - 1) | (1 << (NB - 1))
        return (-v if rng.random() < 0.5 else v), rng.randint(-spread, spread) - NB

    def flip(x, bit):
        v, e = x
        a = abs(v) ^ (1 << bit)
        return (-a if v < 0 else a), e

    # tables with column 1 = -column 0: terms b = 0, 1 cancel where H repeats
    R = [[rnd() for _ in range(S)] for _ in range(S)]
    Q = [[rnd() for _ in range(S)] for _ in range(S)]
    for M in (R, Q):
        for row in M:
            if S >= 2:
                row[1] = (-row[0][0], row[0][1])
    H = [[[[None] * B for _ in range(S)] for _ in range(S)] for _ in range(T)]      # H[t][a][b][k]
    for t in range(T):
        for a in range(S):
            for k in range(B):
                kind = (t + k) % 5
                col = [rnd() for _ in range(S)]
                if kind >= 1 and S >= 2:
                    col[1] = col[0]                                  # exact cancellation of b = 0, 1
                if kind == 2 and S >= 2:
                    col[1] = flip(col[0], rng.randrange(NB - 1))     # cancellation down to a random bit
                if kind == 3 and S >= 2:
                    col[1] = flip(col[0], rng.randrange(NB - 110, NB - 70))   # near the first try's limit
                if kind in (1, 2):
                    col[2:] = [(0, mpf.EZ)] * (S - 2)
                if kind == 4 and S >= 3:
                    col[2] = (col[2][0], col[2][1] - rng.randrange(40, 200))          # a small third term
                for b in range(S):
                    H[t][a][b][k] = col[b]
        for a in range(1, S, 2):                                     # rows a = 1, 3 ... repeat a - 1: stage 2
            for b in range(S):
                for k in range(B):
                    x = H[t][a - 1][b][k]
                    H[t][a][b][k] = x if (a + k) % 3 else (flip(x, rng.randrange(NB - 1)) if x[0] else x)
    return R, Q, H


CASES = [(10, 3, 8, 3, 1), (10, 4, 5, 2, 2), (34, 3, 10, 2, 3), (42, 5, 4, 1, 4)]
MMA_CASES = [(18, 4, 5, 2, 5), (26, 3, 7, 2, 6), (30, 5, 6, 1, 7), (34, 5, 6, 2, 8), (46, 5, 3, 1, 9),
             (34, 2, 40, 1, 10), (22, 6, 20, 1, 11), (38, 8, 3, 1, 12), (14, 1, 9, 2, 13)]


@pytest.mark.parametrize("entry", ["b3d_pole_level", "b3d_pole_level_mma"])
@pytest.mark.parametrize("L,S,B,T,seed", CASES)
def test_pole_step_cancellations_match_exact_sums(cuda, entry, L, S, B, T, seed):
    _run_case(cuda, entry, L, S, B, T, seed)


@pytest.mark.parametrize("L,S,B,T,seed", MMA_CASES)
def test_pole_mma_cancellations_match_exact_sums(cuda, L, S, B, T, seed):
    """every tile geometry of the tensor-core form (one or two tiles of positions, first position 0 to 112),
    column chunks of 16 to 64 with a ragged last chunk (S B = 80, 120), S from 1 to 8"""
    _run_case(cuda, "b3d_pole_level_mma", L, S, B, T, seed)


def _run_case(cuda, entry, L, S, B, T, seed):
    R, Q, H = _case(L, S, B, T, seed)
    flat = lambda M: [x for row in M for x in row]                  # noqa: E731
    Rt = mpf.from_ints(*zip(*flat(R)), L, (1, S, S), cuda)
    Qt = mpf.from_ints(*zip(*flat(Q)), L, (1, S, S), cuda)
    Hflat = [H[t][a][b][k] for t in range(T) for a in range(S) for b in range(S) for k in range(B)]
    Ht = mpf.from_ints(*zip(*Hflat), L, (T, S * S * B), cuda)
    Ra, Qa = mpf.align_rows(Rt), mpf.align_rows(Qt)
    idx = lambda v: torch.tensor(v, dtype=torch.int64, device=cuda)  # noqa: E731
    t_hrow, t_R, t_qL, t_slot = idx(list(range(T))), idx([0] * T), idx([0] * T), idx(list(range(T))[::-1])
    Y = mpf.zeros((T, S * S, B), L, cuda)
    res = mpf.zeros((T, S * S, B), L, cuda)
    p = lambda x: x.data_ptr()                                       # noqa: E731
    args = (L, p(Ht.m), p(Ht.e), Ht.m.stride(0), p(Ra[0]), p(Ra[1]), Ra[0].stride(0),
            p(Qa[0]), p(Qa[1]), Qa[0].stride(0), p(t_hrow), p(t_R), p(t_qL), p(t_slot), T, B, S,
            p(Y.m), p(Y.e), Y.m.stride(0), p(res.m), p(res.e), res.m.stride(0))
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    extra = (p(err),) if entry == "b3d_pole_level_mma" else ()
    _lib.call(entry, *args, *extra, torch.cuda.current_stream(cuda).cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    # Y[t, a, b0, k] = sum_b R[b0, b] H[t, a, b, k];  res[slot(t), a0, b0, k] = sum_a Q[a0, a] Y[t, a, b0, k]
    Yx = {}
    for t in range(T):
        for a in range(S):
            for b0 in range(S):
                for k in range(B):
                    Yx[t, a, b0, k] = _dot(R[b0], [H[t][a][b][k] for b in range(S)], L)
    got_y = mpf.to_ints(Y)
    want_y = [Yx[t, a, b0, k] for t in range(T) for a in range(S) for b0 in range(S) for k in range(B)]
    assert got_y == want_y
    zeros = sum(1 for v, _ in want_y if v == 0)
    if S >= 2:
        assert zeros >= T * S * S * B // 10                          # the exact zeros are really there
    want = {}
    for t in range(T):
        for a0 in range(S):
            for b0 in range(S):
                for k in range(B):
                    want[T - 1 - t, a0, b0, k] = _dot(Q[a0], [Yx[t, a, b0, k] for a in range(S)], L)
    got = mpf.to_ints(res)
    assert got == [want[s, a0, b0, k] for s in range(T) for a0 in range(S) for b0 in range(S) for k in range(B)]
