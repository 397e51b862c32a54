"""Shared builders of the GPU tests: seeded random operators (M matrices, h_inf) as decimal strings, the
h_inf tensor layout of Recursion.run, and the oracle's residues / numerators for the same inputs."""
import random

import mpmath as mp

from blocksvibe_b200 import mpf, plan as PL, structure as S
from oracle import derivatives as OD, recursion as OR


def random_operator(tj12, tj43, tjmax, order, pp, L, nrhs, seed, digits=60):
    """M: key -> matrix of decimal strings (entries uniform in [-2, 2] plus a 2^-150 perturbation, as the
    reference's tests/test_blocks_recursion.py:17); H: [k, src, m, j, a, b, string] for m <= order"""
    rng = random.Random(seed)
    plan = PL.Plan(tj12, tj43, tjmax, order, pp)
    with mp.workprec(32 * L + 64):
        rstr = lambda: mp.nstr(mp.mpf(rng.uniform(-2, 2)) + mp.mpf(rng.random()) * mp.mpf(2) ** -150, digits)
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


def hinf_tensor(entries, plan, order, nrhs, L, device):
    """h_inf MPF (2, order + 1, Jh, S^2, B) from (k, src, m, j, a, b, value string) entries"""
    Sm = plan.Smax
    strs = ["0"] * (2 * (order + 1) * plan.Jh * Sm * Sm * nrhs)
    for k, sp, m, j, a, b, v in entries:
        if m <= order:
            strs[((((sp * (order + 1) + m) * plan.Jh + j) * Sm + a) * Sm + b) * nrhs + k] = v
    return mpf.from_strings(strs, L, (2, order + 1, plan.Jh, Sm * Sm, nrhs), device)


def oracle_residues(M, H, tj12, tj43, tjmax, order, pp, L, k):
    with mp.workprec(32 * L + 64):
        Mn = {key: [[mp.mpf(x) for x in row] for row in v] for key, v in M.items()}
        hk = {(sp, m, j, a, b): mp.mpf(v) for kk, sp, m, j, a, b, v in H if kk == k}
        return OR.fill_residues(hk, Mn, tj12, tj43, tjmax, order, pp), hk


def oracle_numerators(M, H, tj12, tj43, tjmax, order, pp, L, k, R, tjs, kept=None):
    """{(tj, p, a, b): [poly_e for e <= R]} for right-hand side k"""
    res, hk = oracle_residues(M, H, tj12, tj43, tjmax, order, pp, L, k)
    out = {}
    with mp.workprec(32 * L + 64):
        h = lambda p, m, j, a, b: hk.get((p, m, j, a, b), mp.mpf(0))
        r = lambda p, m, j, q, a, b: res.get((p, m, j, q, a, b), mp.mpf(0))
        for tj in tjs:
            for p in range(2):
                for a in range(len(S.so3_structures(pp[p][0], tj12, tj))):
                    for b in range(len(S.so3_structures(pp[p][1], tj43, tj))):
                        out[(tj, p, a, b)] = OD.numerators(h, r, tj, p, a, b, order, R, tj12, tj43, kept)
    return out


def agreement_bits(got, ref):
    """-log2 of max |got - ref| relative to max |ref| (inf when exact, or when ref is all zero and got too)"""
    big = max((abs(x) for x in ref), default=0)
    err = max((abs(g - r) for g, r in zip(got, ref)), default=0)
    if err == 0:
        return float("inf")
    if big == 0:
        return float("-inf")
    return float(-mp.log(err / big, 2))
