"""The drop-in consumer fixture's inputs (shared by make_dropin_golden.py, which runs the reference's cli writer
on them, and the tests): for each spin case of json_cases.py, a group of two blocks_3d invocations (two
four-point structures) given as blocks_3d command lines, and their write_output results as the drop-in returns
them (host limb arrays, seeded values of json_cases.spin_case)."""
import numpy as np

import json_cases as JC


def argv(case, q4, out_dir):
    prec, coords, Lam, sign, pp, tj12, tj43, tjs_int, Dmax, seed = case
    half = lambda t: f"{t / 2:g}"
    return ["--j-external", "1,1,1,1", "--j-internal", ",".join(half(t) for t in tjs_int),
            "--j-12", half(tj12), "--j-43", half(tj43), "--delta-12", "0.25", "--delta-43", "-0.5",
            "--delta-1-plus-2", "2.3", "--four-pt-struct", ",".join(half(t) for t in q4),
            "--four-pt-sign", str(sign), "--order", str(2 * Lam + 6), "--lambda", str(Lam),
            "--coordinates", ",".join(coords), "--kept-pole-order", str(Lam + 3), "--num-threads", "1",
            "--precision", str(prec), "-o", f"{out_dir}/q{''.join(map(str, q4))}_spin_{{}}.json"]


Q4S = ((2, 2, 0, 0), (0, 2, 2, 0))          # doubled four-point structures of the two invocations


def host_values(case):
    """({coord: (m (L, Jo, 2, S^2, 2, outputs, Dmax) int32, e (Jo, 2, S^2, 2, outputs, Dmax) int64)}, outputs,
    Smax, L): task q's values are json_cases.spin_case with seed + 1000 q"""
    prec, coords, Lam, sign, pp, tj12, tj43, tjs_int, Dmax, seed = case
    L = 2 * ((prec + 63) // 64) + 2
    per_task = []
    for q in range(len(Q4S)):
        c2 = case[:-1] + (seed + 1000 * q,)
        _, outputs, Sm, vals = JC.spin_case(c2)
        per_task.append(vals)
    out = {}
    for c in coords:
        nout = len(outputs[c])
        shape = (len(tjs_int), 2, Sm * Sm, len(Q4S), nout, Dmax)
        m = np.zeros((L,) + shape, np.int32)
        e = np.zeros(shape, np.int64)
        for q, vals in enumerate(per_task):
            for jo in range(len(tjs_int)):
                for k in range(2):
                    for s in range(Sm * Sm):
                        for o in range(nout):
                            for d, (v, ex) in enumerate(vals[c][jo][k][s][o]):
                                raw = np.frombuffer(v.to_bytes(4 * L, "little", signed=True), dtype=np.int32)
                                m[:, jo, k, s, q, o, d] = raw
                                e[jo, k, s, q, o, d] = ex if v else -(1 << 60)
        out[c] = (m, e)
    return out, outputs, Sm, L
