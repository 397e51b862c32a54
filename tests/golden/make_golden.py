"""Writes the golden fixtures of tests/golden/ by running the reference's own code (BlocksviBe, read from
REFERENCE below) in this container.  Its GPU modules import cupy / sdpvibe / gmpy2, which are absent
here; empty stand-in modules are registered so that the CPU parts import: structure, recursion_ref (exact
mpmath port of blocks_3d's fill_residues), recursion_gpu.Plan (the index plan), output.Output's
write_output maps, derivatives._shift_columns (pole shifting), and the mpmath ports inside the
reference's tests (tests/test_blocks_derivatives.reference, tests/test_blocks_output.reference_xt).

    python tests/golden/make_golden.py REFERENCE

Fixtures (all seed-fixed):
  plan.npz              Plan tensors for 7 + 1 operator shapes, with and without slot reuse
  recursion.json        random operators / h_inf and the residues of recursion_ref
  derivatives.json      numerators of the reference's mpmath port of residues_to_derivatives ... together
  shift_columns.json    pole-shifting numerator columns of derivatives._shift_columns
  output.json           write_output maps (Output._xt / radial) and reference_xt of random numerators
"""
import json
import os
import random
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) != 2:
    sys.exit(__doc__)
REFERENCE = sys.argv[1]


def _import_reference():
    sys.path.insert(0, REFERENCE)
    sys.path.insert(0, os.path.join(REFERENCE, "tests"))
    for name in ("cupy", "sdpvibe", "sdpvibe.mpf", "sdpvibe.rns", "gmpy2"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["sdpvibe"].mpf = sys.modules["sdpvibe.mpf"]
    sys.modules["sdpvibe"].rns = sys.modules["sdpvibe.rns"]
    sys.modules["sdpvibe.rns"].dev = "cpu"
    sys.modules["sdpvibe.mpf"].MPF = object          # name looked up by the reference's test module


_import_reference()
import mpmath as mp                                                   # noqa: E402
from blocksvibe import structure as S, recursion_ref, recursion_gpu as RG   # noqa: E402
from blocksvibe import derivatives as DV, output as OUT               # noqa: E402

DIGITS = 85


def s(x):
    return mp.nstr(x, DIGITS, strip_zeros=False)


# ---------------------------------------------------------------- plans
PLAN_CASES = [(8, 8, 6, 8, ((0, 0), (1, 1))), (4, 2, 8, 10, ((0, 1), (1, 0))), (3, 1, 9, 12, ((0, 1), (1, 1))),
              (5, 5, 11, 10, ((1, 0), (0, 1))), (4, 4, 6, 9, ((0, 0), (1, 1))), (0, 0, 6, 8, ((0, 0), (1, 1))),
              (8, 4, 4, 7, ((0, 1), (1, 0))), (0, 0, 12, 10, ((0, 0), (1, 1)))]
LEVEL_FIELDS = ("gsrc", "gj", "col", "rowd", "nrow", "cold", "ncol", "t_slot", "t_hrow", "t_L", "t_R", "t_q", "t_qL")


def make_plans():
    out = {}
    for ci, case in enumerate(PLAN_CASES):
        for reuse in (False, True):
            pl = RG.Plan(*case, reuse=reuse)
            k = f"c{ci}_r{int(reuse)}_"
            out[k + "scalars"] = np.array([pl.Smax, pl.Jh, pl.nslots, pl.nphys, pl.zero_slot, pl.dmax], np.int64)
            out[k + "mkeys"] = np.array([[P[0], P[1], d, tjnn, ppq, tj, i] for (P, d, tjnn, ppq, tj), i in pl.Mkeys.items()],
                                        np.int64).reshape(-1, 7)
            out[k + "qkeys"] = np.array([[P[0], P[1], tj, sg, i] for (P, tj, sg), i in pl.Qkeys.items()], np.int64).reshape(-1, 5)
            out[k + "lqpairs"] = np.asarray(pl.LQpairs, np.int64).reshape(-1, 2)
            out[k + "phys"] = np.asarray(pl.phys, np.int64)
            out[k + "levels"] = np.array([-1 if lev is None else lev["m"] for lev in pl.levels], np.int64)
            for lev in pl.levels:
                if lev is None:
                    continue
                m = lev["m"]
                out[k + f"l{m}_dims"] = np.array([lev["nb"], lev["Mr"], lev["Kc"]], np.int64)
                for f in LEVEL_FIELDS:
                    v = lev[f]
                    out[k + f"l{m}_{f}"] = (v.numpy() if hasattr(v, "numpy") else np.asarray(v)).astype(np.int64)
                cd, cx = RG.cauchy_tables(lev)
                out[k + f"l{m}_cdiff"] = cd.numpy().astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "plan.npz"), cases=np.array([list(c[:4]) + [c[4][0][0], c[4][0][1], c[4][1][0], c[4][1][1]]
                                                                         for c in PLAN_CASES], np.int64), **out)


# ---------------------------------------------------------------- recursion
REC_CASES = [  # (tj12, tj43, tj_max, order, pseudo-parities, L, rhs, seed)
    (4, 2, 6, 7, ((0, 1), (1, 0)), 10, 1, 1),
    (8, 8, 4, 5, ((0, 1), (1, 0)), 10, 1, 2),
    (0, 0, 12, 10, ((0, 0), (1, 1)), 10, 1, 3),
    (3, 1, 5, 5, ((0, 1), (1, 1)), 10, 2, 4),
]


def random_operator(tj12, tj43, tj_max, order, pp, L, nrhs, seed):
    """seeded random M matrices (decimal strings, 120 digits) and h_inf for the keys of the operator"""
    rng = random.Random(seed)
    plan = RG.Plan(tj12, tj43, tj_max, order, pp)
    mp.mp.prec = 32 * L + 64
    rstr = lambda: mp.nstr(mp.mpf(rng.uniform(-2, 2)) + mp.mpf(rng.random()) * mp.mpf(2) ** -150, 60)
    M = []
    for (P, d, tjnn, ppq, tj) in plan.Mkeys:
        rows = len(S.so3((ppq + S.parity(P)) % 2, tjnn, tj))
        cols = len(S.so3(ppq, tjnn, S.pole_two_j(P, tj)))
        M.append([[P[0], P[1]], d, tjnn, ppq, tj, [[rstr() for _ in range(cols)] for _ in range(rows)]])
    H = []
    for k in range(nrhs):
        for sp in range(2):
            for m in range(order + 1):
                for j in range(plan.Jh):
                    tj = tj12 % 2 + 2 * j
                    for a in range(len(S.so3(pp[sp][0], tj12, tj))):
                        for b in range(len(S.so3(pp[sp][1], tj43, tj))):
                            H.append([k, sp, m, j, a, b, rstr()])
    return M, H


def make_recursion():
    cases = []
    for (tj12, tj43, tjmax, order, pp, L, nrhs, seed) in REC_CASES:
        M, H = random_operator(tj12, tj43, tjmax, order, pp, L, nrhs, seed)
        mp.mp.prec = 32 * L + 64
        Mn = {((P[0], P[1]), d, tjnn, ppq, tj): [[mp.mpf(x) for x in row] for row in mat] for P, d, tjnn, ppq, tj, mat in M}
        num = lambda x: mp.mpf(x.numerator) / x.denominator if hasattr(x, "numerator") else mp.mpf(x)
        res_all = []
        for k in range(nrhs):
            hk = {(sp, m, j, a, b): mp.mpf(v) for kk, sp, m, j, a, b, v in H if kk == k}
            ref = recursion_ref.recursion(hk, Mn, tj12, tj43, tjmax, order, pp, num)
            res_all += [[k, *key, s(v)] for key, v in sorted(ref.items())]
        cases.append({"tj12": tj12, "tj43": tj43, "tj_max": tjmax, "order": order, "pp": pp, "L": L, "rhs": nrhs,
                      "seed": seed, "M": M, "h_inf": H, "residues": res_all})
    with open(os.path.join(HERE, "recursion.json"), "w") as f:
        json.dump(cases, f)
    return cases


# ---------------------------------------------------------------- derivatives (numerators)
DER_CASES = [(0, 3, None), (3, 0, None), (0, 3, 4)]   # (recursion case index, R, kept pole order)


def make_derivatives(rec_cases):
    import test_blocks_derivatives as TD
    out = []
    for ci, R, kept in DER_CASES:
        c = rec_cases[ci]
        if kept is not None:
            continue                                    # the reference port has no pole shifting
        tj12, tj43, tjmax, order, pp, L = c["tj12"], c["tj43"], c["tj_max"], c["order"], c["pp"], c["L"]
        mp.mp.prec = 32 * L + 64
        hv = {(k, sp, m, j, a, b): mp.mpf(v) for k, sp, m, j, a, b, v in c["h_inf"]}
        rv = {tuple(x[:7]): mp.mpf(x[7]) for x in c["residues"]}
        # the recursion fixture covers levels m < order; h_inf at level `order` enters c[k] too
        polys = []
        for k in range(c["rhs"]):
            h = lambda p, m, j, a, b: hv.get((k, p, m, j, a, b), mp.mpf(0))
            r = lambda p, m, j, q, a, b: rv.get((k, p, m, j, q, a, b), mp.mpf(0))
            for tj in range(tj12 % 2, tjmax + 1, 2):
                for p in range(2):
                    for a in range(len(S.so3(pp[p][0], tj12, tj))):
                        for b in range(len(S.so3(pp[p][1], tj43, tj))):
                            ref = TD.reference(h, r, tj, p, a, b, order, R, tj12, tj43)
                            for e, poly in enumerate(ref):
                                polys.append([k, tj, p, a, b, e, [s(x) for x in poly]])
        out.append({"case": ci, "R": R, "numerators": polys})
    with open(os.path.join(HERE, "derivatives.json"), "w") as f:
        json.dump(out, f)


SHIFT_CASES = [(4, 2, 2, 7, 4), (0, 0, 0, 10, 6), (6, 4, 4, 12, 5), (3, 1, 1, 9, 4)]   # (tj, tj12, tj43, order, kept)


def make_shift_columns():
    """derivatives._shift_columns for some spins: the numerator columns (in y = 2x) of each old pole"""
    out = []
    for tj, tj12, tj43, order, kept in SHIFT_CASES:
        two_ub = tj + 1 if tj <= 1 else tj + 2
        roots = [S.delta_2(P, tj) - two_ub for P in S.poles(tj, tj12, tj43, order)]
        new = [y for y in roots if y == 0] + [S.delta_2(P, tj) - two_ub for P in S.poles(tj, tj12, tj43, kept)
                                              if S.delta_2(P, tj) != two_ub]
        Pi = [1]
        for y0 in new:
            Pi = DV._polymul_lin(Pi, -y0)
        comp = DV._syndiv_all(Pi, new) if new else []
        cols = DV._shift_columns(roots, new, comp, len(new))
        out.append({"tj": tj, "tj12": tj12, "tj43": tj43, "order": order, "kept": kept, "roots": roots, "new": new,
                    "columns": [[i, [str(c) for c in poly], sc, str(den)] for i, poly, sc, den in cols]})
    with open(os.path.join(HERE, "shift_columns.json"), "w") as f:
        json.dump(out, f)


# ---------------------------------------------------------------- write_output
OUT_CASES = [(7, 0, "2.3"), (7, 1, "2.3"), (6, 0, "0"), (9, 1, "6"), (5, 0, "0")]


def make_output():
    import test_blocks_output as TO
    out = []
    L = 10
    for Lam, parity, D in OUT_CASES:
        mp.mp.prec = 32 * L + 128
        o = object.__new__(OUT.Output)
        W = o._xt(Lam, parity, mp.mpf(D))
        O = Lam - parity
        pre = OUT.power_prefactor(O, mp.mpf(D)) if parity == 0 else \
            OUT.one_minus_power_prefactor(O) * OUT.power_prefactor(O, mp.mpf(D) + 1)
        T = pre * OUT.rho_z(O) * OUT.stirling(O)
        rng = random.Random(Lam * 10 + parity)
        nL, R = (Lam - parity) // 2 + 1, Lam - parity
        num = [[mp.mpf(rng.uniform(-1, 1)) * mp.mpf(2) ** rng.randint(-20, 20) if e <= Lam - parity - 2 * idx else mp.mpf(0)
                for e in range(R + 1)] for idx in range(nL)]
        ref = TO.reference_xt(num, Lam, parity, mp.mpf(D))
        out.append({"Lambda": Lam, "parity": parity, "delta_1_plus_2": D, "inputs": o.inputs, "outputs": o.outputs,
                    "W_xt": [[s(x) for x in row] for row in W.tolist()],
                    "T_radial": [[s(T[i, j]) for j in range(T.cols)] for i in range(T.rows)],
                    "num": [[s(x) for x in row] for row in num], "xt": [[s(x) for x in row] for row in ref]})
    with open(os.path.join(HERE, "output.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    make_plans()
    rec = make_recursion()
    make_derivatives(rec)
    make_shift_columns()
    make_output()
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))
