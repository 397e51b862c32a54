"""b3d_pole_level_noalloc, the pole step for callers that cannot allocate device memory while they run (its
scratch is a fixed array inside the library), called through the C ABI and checked against b3d_pole_level
(the same step with a caller-provided scratch buffer) on two calls in a row with different inputs: the
results must be identical, which is within the tolerance of every other test.  Also: a level too large for
the array is refused with B3D_E_ARG and a message, and the refusal leaves the outputs untouched.

Collected last on purpose (file name), so a run stopping at its first failure has run every other test."""
import ctypes

import pytest
import torch

from blocksvibe_b200 import _lib, mpf, plan as PL, recursion as RC

pytestmark = pytest.mark.gpu


def _p(t):
    return t.data_ptr()


def _pole_args(rec, lev, H, res, B):
    Ra, Qa = rec.Ralign, rec.QLalign
    return [_p(H.m), _p(H.e), H.m.stride(0), _p(Ra[0]), _p(Ra[1]), Ra[0].stride(0), _p(Qa[0]), _p(Qa[1]),
            Qa[0].stride(0), _p(lev["t_hrow"]), _p(lev["t_R"]), _p(lev["t_qL"]), _p(lev["t_slot"]), lev["T"], B,
            rec.plan.Smax]


def test_noalloc_pole_level_matches_pole_level(cuda):
    L, B = 10, 2
    plan = PL.Plan(4, 2, 6, 7, ((0, 1), (1, 0)))
    rec = RC.Recursion(plan, None, L, device=cuda, generator=torch.Generator().manual_seed(3))
    S2 = plan.Smax ** 2
    stream = torch.cuda.current_stream(cuda).cuda_stream
    levels = [lev for lev in rec.levels if lev][-2:]
    g = torch.Generator().manual_seed(4)
    lib = _lib.lib()
    for lev in levels:                                          # two calls in a row, different inputs
        H = mpf.random_mpf((rec.max_rows, S2 * B), L, spread=4, device=cuda, generator=g)
        ref = mpf.zeros((plan.nphys + 1, S2, B), L, cuda)
        got = mpf.zeros((plan.nphys + 1, S2, B), L, cuda)
        Y = mpf.zeros((lev["T"], S2, B), L, cuda)
        args = _pole_args(rec, lev, H, ref, B)
        _lib.call("b3d_pole_level", L, *args, _p(Y.m), _p(Y.e), Y.m.stride(0), _p(ref.m), _p(ref.e), ref.m.stride(0), stream)
        rc = lib.b3d_pole_level_noalloc(L, *_pole_args(rec, lev, H, got, B), _p(got.m), _p(got.e), got.m.stride(0), stream)
        assert rc == 0, lib.b3d_last_error().decode()
        torch.cuda.synchronize()
        written = torch.as_tensor(lev["t_slot"]).to(cuda)
        assert (ref.e[written] != mpf.EZ).any()
        assert torch.equal(ref.m, got.m) and torch.equal(ref.e, got.e)


def test_noalloc_rejects_levels_beyond_its_scratch(cuda):
    L, B = 34, 64
    plan = PL.Plan(8, 8, 10, 12, ((0, 0), (1, 1)))
    rec = RC.Recursion(plan, None, L, device=cuda, generator=torch.Generator().manual_seed(5))
    lev = max((lev for lev in rec.levels if lev), key=lambda x: x["T"])
    need = lev["T"] * plan.Smax ** 2 * B * (4 * L + 8)
    assert need > (16 << 20)
    S2 = plan.Smax ** 2
    H = mpf.zeros((rec.max_rows, S2 * B), L, cuda)
    res = mpf.zeros((plan.nphys + 1, S2, B), L, cuda)
    before = res.e.clone()
    lib = _lib.lib()
    rc = lib.b3d_pole_level_noalloc(L, *_pole_args(rec, lev, H, res, B), _p(res.m), _p(res.e), res.m.stride(0),
                                    torch.cuda.current_stream(cuda).cuda_stream)
    assert rc == -2
    assert b"scratch" in lib.b3d_last_error()
    torch.cuda.synchronize()
    assert torch.equal(before, res.e)


def _synthetic_level(cuda, L, S, T, B, rows=64, keys=7, seed=6):
    """random pole-step operands of T tasks (no plan needed): H rows, row-aligned R and q L tables, task maps"""
    g = torch.Generator().manual_seed(seed)
    H = mpf.random_mpf((rows, S * S * B), L, spread=4, device=cuda, generator=g)
    Ra = mpf.align_rows(mpf.random_mpf((keys, S, S), L, spread=2, device=cuda, generator=g))
    Qa = mpf.align_rows(mpf.random_mpf((keys, S, S), L, spread=2, device=cuda, generator=g))
    idx = lambda hi: torch.randint(0, hi, (T,), generator=g).to(cuda)
    return H, Ra, Qa, idx(rows), idx(keys), idx(keys), torch.arange(T, device=cuda)


def test_noalloc_at_its_size_limit(cuda):
    """a level needing exactly B3D_NOALLOC_SCRATCH_BYTES - 256 bytes of scratch (T S^2 B (4 L + 8) with L = 10,
    S = 4, T = 257, B = 85) runs and equals b3d_pole_level bit for bit; one task more is refused"""
    L, S, T, B = 10, 4, 257, 85
    assert T * S * S * B * (4 * L + 8) == (16 << 20) - 256
    H, Ra, Qa, hrow, tR, tq, slot = _synthetic_level(cuda, L, S, T + 1, B)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    lib = _lib.lib()

    def args(n, res):
        return [_p(H.m), _p(H.e), H.m.stride(0), _p(Ra[0]), _p(Ra[1]), Ra[0].stride(0), _p(Qa[0]), _p(Qa[1]),
                Qa[0].stride(0), _p(hrow), _p(tR), _p(tq), _p(slot), n, B, S]
    ref = mpf.zeros((T + 2, S * S, B), L, cuda)
    got = mpf.zeros((T + 2, S * S, B), L, cuda)
    Y = mpf.zeros((T, S * S, B), L, cuda)
    _lib.call("b3d_pole_level", L, *args(T, ref), _p(Y.m), _p(Y.e), Y.m.stride(0), _p(ref.m), _p(ref.e),
              ref.m.stride(0), stream)
    rc = lib.b3d_pole_level_noalloc(L, *args(T, got), _p(got.m), _p(got.e), got.m.stride(0), stream)
    assert rc == 0, lib.b3d_last_error().decode()
    torch.cuda.synchronize()
    assert (ref.e[:T] != mpf.EZ).any()
    assert torch.equal(ref.m, got.m) and torch.equal(ref.e, got.e)
    before = got.e.clone()
    rc = lib.b3d_pole_level_noalloc(L, *args(T + 1, got), _p(got.m), _p(got.e), got.m.stride(0), stream)
    assert rc == -2 and b"scratch" in lib.b3d_last_error()
    torch.cuda.synchronize()
    assert torch.equal(before, got.e)
