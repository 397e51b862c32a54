"""The GPU chain at the benchmark's own sizes against the oracle, through fixtures that the oracle computed
offline (tests/golden/make_chain_golden.py on the inputs of tests/golden/chain_cases.py):

  cfg2_n0      the default bench configuration (2j12 = 2j43 = 8, spins 0-44, order 40, Lambda 11, kept 20,
               1024 bits) at lambda order 0: sampled residue blocks of the slot-recycling recursion (captured
               at their level, before their slots are reused) and the numerator polynomials (R = 11, pole
               shifting) of sampled (spin, parity, structure) blocks;
  cfg5_radial  the largest configuration's shape (order 80, Lambda 27, kept 40, 1280 bits, xt_radial with
               pole shifting) on output spins 0-4: sampled residue blocks, and the xt_radial outputs of sampled
               blocks through the drop-in runner.

Both cases run with each pole-step form: the tensor cores (b3d_pole_level_mma) and the CUDA cores
(b3d_pole_level); with one right-hand side the default form choice would take the CUDA cores, so the form is
forced here.

Bars: residues relative to their (pole, spin) block > 32 L - 64 bits (the reference's recursion bar); every
numerator polynomial and every xt_radial block relative to its largest coefficient > prec - 8 bits (the
drop-in bar).  The worst agreement of each case is printed."""
import gzip
import json
import os
import sys

import mpmath as mp
import pytest
import torch

from conftest import GOLDEN
from helpers import agreement_bits
from blocksvibe_b200 import derivatives as DV, dropin as DI, mpf, plan as PL, recursion as RC, structure as S

sys.path.insert(0, GOLDEN)
import chain_cases as CC                       # noqa: E402

pytestmark = pytest.mark.gpu


def load(name):
    with gzip.open(os.path.join(GOLDEN, f"chain_{name}.json.gz"), "rt") as f:
        return json.load(f)


def m_table(c, plan, device):
    """the case's M matrices as an MPF table (nM, Smax, Smax) in plan.Mkeys order"""
    Sm = plan.Smax
    ints, exps = [0] * (len(plan.Mkeys) * Sm * Sm), [0] * (len(plan.Mkeys) * Sm * Sm)
    for key, i in plan.Mkeys.items():
        r, cc = CC.m_shape(key)
        for a in range(r):
            for b in range(cc):
                ints[(i * Sm + a) * Sm + b], exps[(i * Sm + a) * Sm + b] = CC.m_entry(c["seed"], key, a, b)
    return mpf.from_ints(ints, exps, c["L"], (len(plan.Mkeys), Sm, Sm), device)


def hinf(c, plan, device):
    """h_inf MPF (2, order + 1, Jh, Smax^2) of the case"""
    Sm, order, pp = plan.Smax, c["order"], c["pp"]
    n = 2 * (order + 1) * plan.Jh * Sm * Sm
    ints, exps = [0] * n, [0] * n
    for src in range(2):
        for m in range(order + 1):
            for j in range(plan.Jh):
                tj = c["tj12"] % 2 + 2 * j
                for a in range(len(S.so3_structures(pp[src][0], c["tj12"], tj))):
                    for b in range(len(S.so3_structures(pp[src][1], c["tj43"], tj))):
                        k = (((src * (order + 1) + m) * plan.Jh + j) * Sm + a) * Sm + b
                        ints[k], exps[k] = CC.h_entry(c["seed"], src, m, j, a, b)
    return mpf.from_ints(ints, exps, c["L"], (2, order + 1, plan.Jh, Sm * Sm), device)


def residue_worst(c, fix, plan, captured):
    Sm, bits = plan.Smax, fix["bits"]
    worst = float("inf")
    with mp.workprec(32 * c["L"] + 64):
        for p, m, j, q, ents, E, hx in fix["residues"]:
            ref = CC.decode(E, hx, bits)
            got = captured[(p, m, j, q)]
            g = [got[a * Sm + b] for a, b in ents]
            worst = min(worst, agreement_bits(g, ref))
    return worst


def run_recursion(c, fix, cuda, R=None, pole="auto"):
    """the slot-recycling recursion (and, with R, the moments and numerators) on the case's inputs; the sampled
    residue blocks copied out at their level"""
    plan = PL.Plan(c["tj12"], c["tj43"], c["tjmax"], c["order"], c["pp"], reuse=True)
    rec = RC.Recursion(plan, m_table(c, plan, cuda), c["L"], device=cuda, pole=pole)
    h1 = hinf(c, plan, cuda)
    h = mpf.MPF(h1.m.unsqueeze(-1).contiguous(), h1.e.unsqueeze(-1).contiguous())
    want = {}
    for p, m, j, q, *_ in fix["residues"]:
        want.setdefault(m, []).append((p, m, j, q))
    saved = {}
    der = None
    if R is not None:
        der = DV.Derivs(plan, R, c["L"], kept_pole_order=c["kept"], device=cuda)
        der.start(1)

    def hook(m, res):
        for key in want.get(m, []):
            p, _, j, q = key
            slot = plan.phys_slot(p * plan.nslots + plan.offset(m, j) + q)
            saved[key] = mpf.MPF(res.m[:, slot, :, 0].clone(), res.e[slot, :, 0].clone())
        if der is not None:
            der.accumulate(m, res)

    rec.run(h, hook=hook)
    num = der.finish(h) if der is not None else None
    torch.cuda.synchronize()
    rec.check_errors()
    captured = {k: mpf.to_mp(v) for k, v in saved.items()}
    return plan, der, num, captured, h1


@pytest.mark.parametrize("pole", ["mma", "cuda"])
def test_cfg2_lambda0_residues_and_numerators(cuda, pole):
    fix = load("cfg2_n0")
    c = CC.CASES["cfg2_n0"]
    R = c["Lam"] - c["n"]
    plan, der, num, captured, _ = run_recursion(c, fix, cuda, R=R, pole=pole)
    rw = residue_worst(c, fix, plan, captured)
    num = mpf.to_mp(num)                                  # (Jo, Dout, R + 1, 2, S^2, 1)
    Sm, bits = plan.Smax, fix["bits"]
    worst, count = float("inf"), 0
    with mp.workprec(32 * c["L"] + 64):
        for (tj, p, a, b), polys in fix["outputs"]:
            jo = der.tjs.index(tj)
            for e, (E, hx) in enumerate(polys):
                ref = CC.decode(E, hx, bits)
                assert len(ref) <= der.Dout
                ref = ref + [mp.mpf(0)] * (der.Dout - len(ref))
                if max(abs(x) for x in ref) == 0:
                    continue
                g = [num[jo, i, e, p, a * Sm + b, 0] for i in range(der.Dout)]
                worst = min(worst, agreement_bits(g, ref))
                count += 1
    print(f"\ncfg2 lambda order 0, pole step {pole}: residues {rw:.1f} bits over {len(fix['residues'])} blocks (bar {32 * c['L'] - 64}); "
          f"numerators {worst:.1f} bits over {count} polynomials (bar {c['precision'] - 8})")
    assert count > 0
    assert rw > 32 * c["L"] - 64, rw
    assert worst > c["precision"] - 8, worst


@pytest.mark.parametrize("pole", ["mma", "cuda"])
def test_cfg5_shape_radial_with_pole_shifting(cuda, pole, monkeypatch):
    fix = load("cfg5_radial")
    c = CC.CASES["cfg5_radial"]
    monkeypatch.setattr(RC, "POLE", pole)                 # the drop-in runner's recursions too
    plan, _, _, captured, h1 = run_recursion(c, fix, cuda, pole=pole)
    rw = residue_worst(c, fix, plan, captured)
    G = DI.Group((4, 4, 4, 4), c["tj12"], c["tj43"], c["order"], c["Lam"], c["tjmax"], c["precision"], c["kept"])
    tjs = list(range(c["tj12"] % 2, c["tjmax"] + 1, 2))
    t = DI.Task((0, 0, 0, 0), 1, c["pp"], tjs, (c["coord"],), c["d12"])
    t.h_inf[c["n"]] = mpf.MPF(h1.m.cpu(), h1.e.cpu())
    res = DI.run_group(G, [t], {c["pp"]: m_table(c, plan, cuda)}, device=cuda, schedule="plain")
    got_tjs, _, vals, _, Smax, _ = res[(t.q4, t.sign)]
    m, e = vals[(c["coord"], c["d12"])]                  # (L, Jo, 2, S^2, outputs, Dmax)
    got = mpf.to_mp(mpf.MPF(torch.from_numpy(m), torch.from_numpy(e)))
    bits = fix["bits"]
    worst, count = float("inf"), 0
    with mp.workprec(32 * c["L"] + 64):
        for (tj, p, a, b), polys in fix["outputs"]:
            jo = got_tjs.index(tj)
            Dmax = got.shape[-1]
            assert len(polys) == got.shape[-2]
            for o, (E, hx) in enumerate(polys):
                ref = CC.decode(E, hx, bits)
                assert len(ref) <= Dmax
                ref = ref + [mp.mpf(0)] * (Dmax - len(ref))
                if max(abs(x) for x in ref) == 0:
                    continue
                g = [got[jo, p, a * Smax + b, o, d] for d in range(Dmax)]
                worst = min(worst, agreement_bits(g, ref))
                count += 1
    print(f"\ncfg5 shape xt_radial, pole step {pole}: residues {rw:.1f} bits over {len(fix['residues'])} blocks (bar {32 * c['L'] - 64}); "
          f"xt_radial outputs {worst:.1f} bits over {count} polynomials (bar {c['precision'] - 8})")
    assert count > 0
    assert rw > 32 * c["L"] - 64, rw
    assert worst > c["precision"] - 8, worst
