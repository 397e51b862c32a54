"""GPU radial recursion (libb3dgpu.so through blocksvibe_b200.recursion) against the oracle's
fill_residues on the same operators and initial data: the reference's own bar (its
tests/test_blocks_recursion.py:52), error relative to each (pole, spin) block > 32 L - 64 bits."""
import random

import mpmath as mp
import pytest
import torch

from conftest import golden, golden_operator
from blocksvibe_b200 import mpf, plan as PL, recursion as RC, structure as S
from oracle import recursion as OR

pytestmark = pytest.mark.gpu


def hinf_tensor(entries, plan, order, nrhs, L, device):
    """h_inf MPF (2, order + 1, Jh, S^2, B) from (k, src, m, j, a, b, value string) entries"""
    Sm = plan.Smax
    strs = ["0"] * (2 * (order + 1) * plan.Jh * Sm * Sm * nrhs)
    for k, sp, m, j, a, b, v in entries:
        strs[((((sp * (order + 1) + m) * plan.Jh + j) * Sm + a) * Sm + b) * nrhs + k] = v
    return mpf.from_strings(strs, L, (2, order + 1, plan.Jh, Sm * Sm, nrhs), device)


def random_case(tj12, tj43, tjmax, order, pp, L, nrhs, seed):
    rng = random.Random(seed)
    plan = PL.Plan(tj12, tj43, tjmax, order, pp)
    mp.mp.prec = 32 * L + 64
    rstr = lambda: mp.nstr(mp.mpf(rng.uniform(-2, 2)) + mp.mpf(rng.random()) * mp.mpf(2) ** -150, 60)
    M = {}
    for (P, d, tjnn, ppq, tj) in plan.Mkeys:
        rows = len(S.so3_structures((ppq + S.pole_parity(P)) % 2, tjnn, tj))
        cols = len(S.so3_structures(ppq, tjnn, S.child_spin(P, tj)))
        M[(P, d, tjnn, ppq, tj)] = [[rstr() for _ in range(cols)] for _ in range(rows)]
    H = []
    for k in range(nrhs):
        for sp in range(2):
            for m in range(order + 1):
                for j in range(plan.Jh):
                    tj = tj12 % 2 + 2 * j
                    for a in range(len(S.so3_structures(pp[sp][0], tj12, tj))):
                        for b in range(len(S.so3_structures(pp[sp][1], tj43, tj))):
                            H.append([k, sp, m, j, a, b, rstr()])
    return M, H


def check(tj12, tj43, tjmax, order, pp, L, nrhs, M, H, device, reuse=False, cauchy="auto"):
    plan = PL.Plan(tj12, tj43, tjmax, order, pp, reuse=reuse)
    rec = RC.Recursion(plan, M, L, device=device, cauchy=cauchy)
    res = mpf.to_mp(rec.run(hinf_tensor(H, plan, order, nrhs, L, device)))
    mp.mp.prec = 32 * L + 64
    Mn = {k: [[mp.mpf(x) for x in row] for row in v] for k, v in M.items()}
    Sm = plan.Smax
    worst = mp.inf
    count = 0
    for k in range(nrhs):
        hk = {(sp, m, j, a, b): mp.mpf(v) for kk, sp, m, j, a, b, v in H if kk == k}
        ref = OR.fill_residues(hk, Mn, tj12, tj43, tjmax, order, pp)
        block = {}
        for key, v in ref.items():
            block[key[:4]] = max(block.get(key[:4], 0), abs(v))
        for (p, m, j, q, a, b), v in ref.items():
            slot = plan.phys_slot(p * plan.nslots + plan.offset(m, j) + q)
            g = res[slot, a * Sm + b, k]
            if block[(p, m, j, q)]:
                err = abs(g - v) / block[(p, m, j, q)]
                worst = min(worst, -mp.log(err, 2) if err else mp.inf)
                count += 1
    assert count > 0
    assert worst > 32 * L - 64, (float(worst), count)
    return float(worst)


@pytest.mark.parametrize("cauchy", ["cuda", "rns"])
@pytest.mark.parametrize("ci", range(4))
def test_recursion_golden_operators(cuda, ci, cauchy):
    c = golden("recursion.json")[ci]
    M, H = golden_operator(c)
    check(c["tj12"], c["tj43"], c["tj_max"], c["order"], tuple(tuple(x) for x in c["pp"]), c["L"], c["rhs"], M, H, cuda,
          cauchy=cauchy)


@pytest.mark.parametrize("case", [
    (4, 2, 6, 7, ((0, 1), (1, 0)), 10, 3, 11),
    (8, 8, 4, 6, ((0, 1), (1, 0)), 10, 2, 12),
    (3, 1, 5, 6, ((0, 1), (1, 1)), 18, 2, 13),
    (2, 2, 6, 8, ((0, 0), (1, 1)), 34, 1, 14),
])
@pytest.mark.parametrize("cauchy", ["cuda", "cuda3", "rns"])
def test_recursion_random_operators(cuda, case, cauchy):
    tj12, tj43, tjmax, order, pp, L, nrhs, seed = case
    M, H = random_case(*case)
    check(tj12, tj43, tjmax, order, pp, L, nrhs, M, H, cuda, cauchy=cauchy)


def test_slot_reuse_same_live_residues(cuda):
    """recycled slots: every residue that is still live at the end equals the run without reuse"""
    case = (4, 2, 6, 8, ((0, 1), (1, 0)), 10, 2, 21)
    M, H = random_case(*case)
    tj12, tj43, tjmax, order, pp, L, nrhs, _ = case
    a = PL.Plan(tj12, tj43, tjmax, order, pp, reuse=False)
    b = PL.Plan(tj12, tj43, tjmax, order, pp, reuse=True)
    ra = RC.Recursion(a, M, L, device=cuda).run(hinf_tensor(H, a, order, nrhs, L, cuda))
    rb = RC.Recursion(b, M, L, device=cuda).run(hinf_tensor(H, b, order, nrhs, L, cuda))
    last = [lev for lev in a.levels if lev][-1]
    # residues of the last level are written last: no later level can recycle their slots
    for t in range(len(last["t_slot"])):
        la = int(last["t_slot"][t])
        logical = int(torch.nonzero(torch.as_tensor(a.phys) == la)[0])
        lb = b.phys_slot(logical)
        assert torch.equal(ra.m[:, la], rb.m[:, lb]) and torch.equal(ra.e[la], rb.e[lb])


@pytest.mark.parametrize("case", [
    (4, 2, 6, 9, ((0, 1), (1, 0)), 10, 3, 61),              # divisors < 2^8: 24-bit digits in cuda3
    (8, 8, 6, 8, ((0, 0), (1, 1)), 34, 2, 62),
    (2, 2, 60, 50, ((0, 0), (1, 1)), 10, 1, 63),            # divisors up to 314: 22-bit digits in cuda3
])
def test_cauchy_forms_bitwise_equal(cuda, case):
    """the pre-aligned two-terms-per-thread Cauchy kernel, its wide-digit form and the wide-digit form on
    sign-magnitude columns read limb by limb give the first kernel's bits"""
    tj12, tj43, tjmax, order, pp, L, nrhs, seed = case
    M, H = random_case(*case)
    plan = PL.Plan(tj12, tj43, tjmax, order, pp, reuse=True)
    outs = []
    for form in ("cuda", "cuda2", "cuda3", "cuda4"):
        rec = RC.Recursion(plan, M, L, device=cuda, cauchy=form)
        outs.append(rec.run(hinf_tensor(H, plan, order, nrhs, L, cuda)))
    for o in outs[1:]:
        assert torch.equal(outs[0].m, o.m) and torch.equal(outs[0].e, o.e)


@pytest.mark.parametrize("case", [
    (4, 2, 6, 9, ((0, 1), (1, 0)), 10, 3, 71),
    (8, 8, 6, 8, ((0, 0), (1, 1)), 34, 2, 72),
    (4, 4, 8, 8, ((0, 0), (1, 1)), 26, 5, 73),
    (8, 8, 6, 6, ((0, 1), (1, 0)), 42, 3, 74),
    (8, 8, 4, 6, ((0, 0), (1, 1)), 46, 14, 75),             # S B = 70 columns: two column chunks
])
def test_pole_forms_bitwise_equal(cuda, case):
    """the pole step's exact sums on the tensor cores (b3d_pole_level_mma) give the CUDA-core kernels' bits
    over a whole recursion with slot recycling, and the residues meet the oracle's bar"""
    tj12, tj43, tjmax, order, pp, L, nrhs, seed = case
    M, H = random_case(*case)
    plan = PL.Plan(tj12, tj43, tjmax, order, pp, reuse=True)
    outs = []
    for form in ("cuda", "mma"):
        rec = RC.Recursion(plan, M, L, device=cuda, pole=form)
        outs.append(rec.run(hinf_tensor(H, plan, order, nrhs, L, cuda)))
        rec.check_errors()
    assert torch.equal(outs[0].m, outs[1].m) and torch.equal(outs[0].e, outs[1].e)
    check(tj12, tj43, tjmax, order, pp, L, nrhs, M, H, cuda)
