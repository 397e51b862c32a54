"""GPU post-recursion stages and write_output against the oracle: numerator polynomials (moments accumulated
during a slot-recycling recursion, residues a, G, polynomial part, numerator GEMM; with and without pole
shifting) and the xt / xt_radial maps applied on the GPU.  The reference's bar: error relative to the largest
coefficient of each polynomial > 32 L - 40 bits (its tests/test_blocks_derivatives.py:118,
tests/test_blocks_output.py:75)."""
import random

import mpmath as mp
import pytest
import torch

from helpers import agreement_bits, hinf_tensor, oracle_numerators, random_operator
from blocksvibe_b200 import derivatives as DV, mpf, output as OUT, plan as PL, recursion as RC
from oracle import output as OO

pytestmark = pytest.mark.gpu


def run_numerators(case, device, R, kept=None, chunk=2):
    tj12, tj43, tjmax, order, pp, L, nrhs, seed = case
    M, H = random_operator(*case)
    plan = PL.Plan(tj12, tj43, tjmax, order, pp, reuse=True)
    rec = RC.Recursion(plan, M, L, device=device)
    der = DV.Derivs(plan, R, L, kept_pole_order=kept, device=device)
    h = hinf_tensor(H, plan, order, nrhs, L, device)
    der.start(nrhs)
    rec.run(h, hook=der.accumulate)
    num = mpf.to_mp(der.finish(h, chunk=chunk))
    return M, H, plan, der, num


def compare_numerators(case, M, H, plan, der, num, R, kept=None):
    tj12, tj43, tjmax, order, pp, L, nrhs, _ = case
    Sm = plan.Smax
    worst, count = float("inf"), 0
    for k in range(nrhs):
        ref = oracle_numerators(M, H, tj12, tj43, tjmax, order, pp, L, k, R, der.tjs, kept)
        for (tj, p, a, b), polys in ref.items():
            jo = der.tjs.index(tj)
            for e, poly in enumerate(polys):
                g = [num[jo, i, e, p, a * Sm + b, k] for i in range(der.Dout)]
                assert len(poly) <= der.Dout
                poly = list(poly) + [mp.mpf(0)] * (der.Dout - len(poly))
                bits = agreement_bits(g, poly)
                if max(abs(x) for x in poly) == 0:
                    continue
                worst = min(worst, bits)
                count += 1
    assert count > 0
    assert worst > 32 * L - 40, (worst, count)
    return worst


@pytest.mark.parametrize("case,R", [
    ((4, 2, 6, 7, ((0, 1), (1, 0)), 10, 2, 31), 3),
    ((8, 8, 4, 6, ((0, 1), (1, 0)), 10, 1, 32), 5),
    ((3, 1, 5, 5, ((0, 1), (1, 1)), 10, 2, 33), 0),
    ((2, 2, 4, 8, ((0, 0), (1, 1)), 18, 1, 34), 4),
])
def test_numerators_match_oracle(cuda, case, R):
    M, H, plan, der, num = run_numerators(case, cuda, R)
    compare_numerators(case, M, H, plan, der, num, R)


@pytest.mark.parametrize("case,R,kept", [
    ((2, 2, 4, 9, ((0, 0), (1, 1)), 10, 1, 41), 3, 4),
    ((4, 2, 6, 8, ((0, 1), (1, 0)), 10, 1, 42), 2, 5),
])
def test_pole_shifted_numerators_match_oracle(cuda, case, R, kept):
    M, H, plan, der, num = run_numerators(case, cuda, R, kept=kept)
    compare_numerators(case, M, H, plan, der, num, R, kept=kept)


@pytest.mark.parametrize("mode,stage_bytes", [("staged", 1 << 40), ("staged", 1), ("per_level", 1 << 40)])
def test_moment_modes_match_oracle(cuda, mode, stage_bytes, monkeypatch):
    """the staged moments with one window for the whole recursion, with a one-level window (a flush and an
    addition into the moments at every level), and the per-level read-modify-write: numerators against the oracle"""
    monkeypatch.setattr(DV, "MOMENTS", mode)
    monkeypatch.setattr(DV, "STAGE_BYTES", stage_bytes)
    case, R, kept = (4, 2, 6, 9, ((0, 1), (1, 0)), 10, 2, 61), 4, 6
    M, H, plan, der, num = run_numerators(case, cuda, R, kept=kept)
    compare_numerators(case, M, H, plan, der, num, R, kept=kept)


def test_staged_window_sums_cancel_exactly(cuda, monkeypatch):
    """the flush's window sum is exact: staged terms y = (x, -2 x, x) at n = (s, s + 1, s + 2) (a second difference)
    give exact zeros for the moments of order 0 and 1 and the correctly rounded sum for the higher orders"""
    L, order, R = 10, 6, 3
    plan = PL.Plan(0, 0, 2, order, ((0, 0), (1, 1)), reuse=True)
    der = DV.Derivs(plan, R, L, device=cuda)
    rows, N = 2 * der.Jo * der.NP, 3
    W = 3
    with mp.workprec(32 * L + 64):
        x = mp.mpf(3) / 7
        s = int(der._row_shift[0])                       # row 0's pole: n = w + s at window level w
        n = [w + s for w in range(W)]
        y = [x, -2 * x, x]
        vals = []
        for w in range(W):
            for r in range(rows):
                for c in range(N):
                    vals.append(y[w] if r == 0 else mp.mpf(0))
    stage = mpf.from_mp(vals, L, (W, rows, N), cuda)
    mom = mpf.zeros((rows, R + 1, N), L, cuda)
    p = lambda t: t.data_ptr()
    from blocksvibe_b200 import _lib
    _lib.call("b3d_moments_flush", L, p(stage.m), p(stage.e), stage.m.stride(0), p(der._row_shift), 0, W, rows, N, R + 1,
              p(der._nk[:R + 1].contiguous()), p(der._nkb[:R + 1].contiguous()), order + 1, der._KW, 0, L, p(mom.m),
              p(mom.e), mom.m.stride(0), torch.cuda.current_stream(cuda).cuda_stream)
    got = mpf.to_mp(mom)
    with mp.workprec(32 * L + 200):
        for k in range(R + 1):
            want = mp.fsum(mp.mpf(nn) ** k * yy for nn, yy in zip(n, y))
            for c in range(N):
                if want == 0:
                    assert got[0, k, c] == 0
                else:
                    assert abs(got[0, k, c] - want) <= abs(want) * mp.mpf(2) ** (2 - (32 * L - 2))
        assert all(v == 0 for v in got[1:].reshape(-1))


def test_for_order_views(cuda):
    """Derivs.for_order(R') (a higher lambda order) gives the numerators of a Derivs built for R'"""
    case = (2, 2, 4, 7, ((0, 0), (1, 1)), 10, 1, 51)
    tj12, tj43, tjmax, order, pp, L, nrhs, seed = case
    M, H = random_operator(*case)
    plan = PL.Plan(tj12, tj43, tjmax, order, pp, reuse=True)
    rec = RC.Recursion(plan, M, L, device=cuda)
    h = hinf_tensor(H, plan, order, nrhs, L, cuda)
    big = DV.Derivs(plan, 5, L, device=cuda).for_order(2)
    small = DV.Derivs(plan, 2, L, device=cuda)
    outs = []
    for d in (big, small):
        d.start(nrhs)
        rec.run(h, hook=d.accumulate)
        outs.append(d.finish(h))
    assert outs[0].shape == outs[1].shape
    assert torch.equal(outs[0].m, outs[1].m) and torch.equal(outs[0].e, outs[1].e)


@pytest.mark.parametrize("Lam,parity,D", [(7, 0, "2.3"), (7, 1, "2.3"), (6, 0, "0"), (9, 1, "6")])
def test_write_output_on_gpu(cuda, Lam, parity, D):
    L = 10
    rng = random.Random(Lam * 7 + parity)
    o_xt, o_rad = OUT.Output("xt", Lam, parity, D, L, cuda), OUT.Output("xt_radial", Lam, parity, D, L, cuda)
    nL, R = (Lam - parity) // 2 + 1, Lam - parity
    with mp.workprec(32 * L + 128):
        num = [[mp.mpf(rng.uniform(-1, 1)) * mp.mpf(2) ** rng.randint(-20, 20) if e <= R - 2 * idx else mp.mpf(0)
                for e in range(R + 1)] for idx in range(nL)]
        vals = [num[idx][e] if p == 0 else mp.mpf(0) for e in range(R + 1) for p in range(2) for idx in range(nL)]
        X = mpf.from_mp(vals, L, (1, 1, R + 1, 2, 1, nL), cuda)
        for o, ref in ((o_xt, [x for row in OO.xt(num, Lam, parity, D) for x in row]),
                       (o_rad, OO.xt_radial(num[0], Lam, parity, D))):
            got = list(mpf.to_mp(o.apply(X, nL=nL))[0, 0, 0, 0, :, 0])
            assert agreement_bits(got, ref) > 32 * L - 40


@pytest.mark.parametrize("L", [10, 34, 42])
def test_resize_widens_exactly_and_narrows_once(cuda, L):
    """b3d_resize: L -> L + 4 keeps every value, L + 4 -> L rounds once as the host conversions round"""
    g = torch.Generator().manual_seed(L)
    X = mpf.random_mpf((300,), L, spread=30, device=cuda, generator=g)
    X.m[:, 0] = 0
    X.e[0] = mpf.EZ
    W = DV.resize(X, L + 4)
    assert W.L == L + 4
    assert list(mpf.to_mp(W)) == list(mpf.to_mp(X))
    back = DV.resize(W, L)
    assert torch.equal(back.m, X.m) and torch.equal(back.e, X.e)
    Y = mpf.random_mpf((300,), L + 4, spread=30, device=cuda, generator=g)
    got = mpf.to_mp(DV.resize(Y, L))
    with mp.workprec(32 * (L + 4) + 64):
        want = mpf.to_mp(mpf.from_mp(list(mpf.to_mp(Y)), L))
    assert list(got) == list(want)
