"""The drop-in group runner end to end (recursion -> numerators per lambda order -> xt / xt_radial) against
the oracle chain (fill_residues -> numerators -> write_output transforms), and the schedules against each
other: the batched pass (all structures and lambda orders as one batch) gives the plain per-order results
bit for bit, and a task's result is the same alone and in a mix with other tasks."""
import random

import mpmath as mp
import numpy as np
import pytest
import torch

from helpers import agreement_bits, oracle_numerators
from blocksvibe_b200 import dropin as DI, mpf, plan as PL, recursion as RC, structure as S
from oracle import output as OO

pytestmark = pytest.mark.gpu


def make_group(tj12=2, tj43=2, tjmax=4, order=8, Lam=4, precision=256, kept=5, seed=7, nq=2,
               coords=("xt", "xt_radial"), sign=1, pp=((0, 0), (1, 1)), d12="2.3"):
    G = DI.Group((2, 2, 2, 2), tj12, tj43, order, Lam, tjmax, precision, kept)
    L = DI.limbs(precision)
    plan = PL.Plan(tj12, tj43, tjmax, order, pp)
    rng = random.Random(seed)
    digits = 32 * L // 3
    with mp.workprec(32 * L + 64):
        rstr = lambda: mp.nstr(mp.mpf(rng.uniform(-2, 2)) + mp.mpf(rng.random()) * mp.mpf(2) ** -150, digits)
        M = {key: [[rstr() for _ in range(len(S.so3_structures(key[3], key[2], S.child_spin(key[0], key[4]))))]
                   for _ in range(len(S.so3_structures((key[3] + S.pole_parity(key[0])) % 2, key[2], key[4])))]
             for key in plan.Mkeys}
        Sm = plan.Smax
        tasks, hstr = [], {}
        for q in range(nq):
            t = DI.Task((q, 2, 2 - q, 0), sign, pp, list(range(0, tjmax + 1, 2)), coords, d12)
            for n in t.lambda_orders(Lam):
                strs = ["0"] * (2 * (order + 1) * plan.Jh * Sm * Sm)
                ent = []
                for sp in range(2):
                    for m in range(order + 1):
                        for j in range(plan.Jh):
                            tj = tj12 % 2 + 2 * j
                            for a in range(len(S.so3_structures(pp[sp][0], tj12, tj))):
                                for b in range(len(S.so3_structures(pp[sp][1], tj43, tj))):
                                    v = rstr()
                                    strs[(((sp * (order + 1) + m) * plan.Jh + j) * Sm + a) * Sm + b] = v
                                    ent.append([0, sp, m, j, a, b, v])
                t.h_inf[n] = mpf.from_strings(strs, L, (2, order + 1, plan.Jh, Sm * Sm))
                hstr[(q, n)] = ent
            tasks.append(t)
    return G, tasks, M, hstr, plan


def test_dropin_matches_oracle_chain(cuda):
    worst = chain_worst_bits(cuda, *make_group())
    assert worst > 32 * DI.limbs(256) - 40, worst


@pytest.mark.parametrize("name,args", [
    ("cfg1", dict(tj12=0, tj43=0, tjmax=12, order=10, Lam=5, precision=256, kept=6, nq=1, coords=("xt",))),
    ("cfg1_radial_odd", dict(tj12=0, tj43=0, tjmax=12, order=10, Lam=5, precision=256, kept=6, nq=1,
                             coords=("xt_radial",), sign=-1)),
    ("cfg2_shape_512", dict(tj12=8, tj43=8, tjmax=8, order=8, Lam=5, precision=512, kept=5, nq=1, coords=("xt",))),
    ("cfg2_shape_1024", dict(tj12=8, tj43=8, tjmax=4, order=6, Lam=3, precision=1024, kept=4, nq=1, coords=("xt",))),
    # the other limb counts the benchmarks run: 768 / 896 bits (644-task set, L = 26 / 30) and 1280 bits (serving
    # stream and largest configuration, L = 42), each with pole shifting and both coordinates
    ("set644_768", dict(tj12=4, tj43=4, tjmax=4, order=8, Lam=5, precision=768, kept=5, nq=1,
                        coords=("xt", "xt_radial"), d12="0.7")),
    ("set644_896_odd", dict(tj12=2, tj43=2, tjmax=6, order=8, Lam=5, precision=896, kept=6, nq=1,
                            coords=("xt", "xt_radial"), sign=-1, pp=((0, 1), (1, 0)))),
    ("cfg5_1280", dict(tj12=8, tj43=8, tjmax=4, order=7, Lam=4, precision=1280, kept=5, nq=1,
                       coords=("xt", "xt_radial"), d12="6")),
])
@pytest.mark.parametrize("pole", ["cuda", "mma"])
def test_worst_bits_per_config(cuda, name, args, pole, monkeypatch):
    """the drop-in bar (blocks_3d's outputs to 2^-(prec - 8)): every output agrees with the oracle chain to more
    than prec - 8 bits (relative to each polynomial's largest coefficient); the worst case is printed per
    configuration and pole-step form (the tensor cores, or the CUDA cores)"""
    monkeypatch.setattr(RC, "POLE", pole)
    G, tasks, M, hstr, plan = make_group(**args)
    worst = chain_worst_bits(cuda, G, tasks, M, hstr, plan)
    print(f"\nworst-case agreement {name}, pole step {pole}: {worst:.1f} bits (precision {G.precision}, "
          f"NB {32 * DI.limbs(G.precision) - 2})")
    assert worst > G.precision - 8, worst


def chain_worst_bits(cuda, G, tasks, M, hstr, plan):
    L = DI.limbs(G.precision)
    res = DI.run_group(G, tasks, M, device=cuda, schedule="plain")
    Sm = plan.Smax
    t0 = tasks[0]
    tjs, pp, vals, outputs, Smax, NB = res[(tuple(t0.q4), t0.sign)]
    assert NB == 32 * L - 2 and Smax == Sm
    ns = t0.lambda_orders(G.Lambda)
    nums = {n: oracle_numerators(M, hstr[(0, n)], G.two_j12, G.two_j43, G.two_j_max, G.order, t0.pp, L, 0,
                                 G.Lambda - n, tjs, G.kept_pole_order) for n in ns}
    got = {}
    for c in t0.coordinates:
        m, e = vals[(c, t0.delta_1_plus_2)]
        got[c] = mpf.to_mp(mpf.MPF(torch.from_numpy(m), torch.from_numpy(e)))      # (Jo, 2, S2, outputs, Dmax)
    worst = float("inf")
    with mp.workprec(32 * L + 128):
        for (tj, p, a, b), _ in nums[ns[0]].items():
            jo = tjs.index(tj)
            Dmax = next(iter(got.values())).shape[-1]
            for dcoef in range(Dmax):
                # num[idx][e] for coefficient dcoef
                table = []
                for n in ns:
                    polys = nums[n][(tj, p, a, b)]
                    table.append([polys[ee][dcoef] if ee <= G.Lambda - n and dcoef < len(polys[ee]) else mp.mpf(0)
                                  for ee in range(G.Lambda - t0.parity + 1)])
                refs = {}
                if "xt" in got:
                    refs["xt"] = [x for row in OO.xt(table, G.Lambda, t0.parity, t0.delta_1_plus_2) for x in row]
                if "xt_radial" in got:
                    refs["xt_radial"] = OO.xt_radial(table[0], G.Lambda, t0.parity, t0.delta_1_plus_2)
                for c, r in refs.items():
                    if max(abs(x) for x in r) == 0:
                        continue
                    g = [got[c][jo, p, a * Sm + b, o, dcoef] for o in range(len(r))]
                    worst = min(worst, agreement_bits(g, r))
    return float(worst)


def test_batched_schedule_is_bitwise_plain(cuda):
    G, tasks, M, _, _ = make_group(nq=3, seed=9, coords=("xt",))
    a = DI.run_group(G, tasks, M, device=cuda, schedule="plain")
    b = DI.run_group(G, tasks, M, device=cuda, schedule="batched")
    assert a.keys() == b.keys()
    for k in a:
        for c in a[k][2]:
            assert np.array_equal(a[k][2][c][0], b[k][2][c][0]) and np.array_equal(a[k][2][c][1], b[k][2][c][1])


def test_result_same_alone_and_in_mix(cuda):
    G, tasks, M, _, _ = make_group(nq=3, seed=11, coords=("xt",), sign=-1)
    mix = DI.run_group(G, tasks, M, device=cuda, schedule="batched")
    alone = DI.run_group(G, tasks[1:2], M, device=cuda, schedule="batched")
    k = (tuple(tasks[1].q4), tasks[1].sign)
    for c in alone[k][2]:
        assert np.array_equal(alone[k][2][c][0], mix[k][2][c][0]) and np.array_equal(alone[k][2][c][1], mix[k][2][c][1])


def test_cuda_graph_step_equals_launched_step(cuda):
    """the captured step, replayed on two different batches, gives the launched step's bits"""
    G, tasks, M, _, _ = make_group(nq=2, seed=31, coords=("xt", "xt_radial"))
    t = tasks[0]
    ns = t.lambda_orders(G.Lambda)
    op = DI.Operator(G, t.pp, t.parity, M, t.two_js_internal, list(t.coordinates), [t.delta_1_plus_2], cuda)
    g = DI.GraphStep(op, 1, ns, t.delta_1_plus_2)
    for task in tasks:
        ref = op.apply_outputs(op.run_batched([task], ns), t.delta_1_plus_2)
        got = g.run([task])
        for c in ref:
            assert torch.equal(ref[c].m, got[c].m) and torch.equal(ref[c].e, got[c].e), c


def test_pipelined_stream_equals_replays(cuda):
    """run_stream (inputs in and results out on a copy stream, overlapping the next replay) yields, batch by batch,
    the bits of separate replays, also when a batch repeats and the double buffers wrap around"""
    import dataclasses
    G, tasks, M, _, _ = make_group(nq=3, seed=37, coords=("xt", "xt_radial"))
    t = tasks[0]
    ns = t.lambda_orders(G.Lambda)
    op = DI.Operator(G, t.pp, t.parity, M, t.two_js_internal, list(t.coordinates), [t.delta_1_plus_2], cuda)
    g = DI.GraphStep(op, 1, ns, t.delta_1_plus_2)
    seq = [tasks[0], tasks[1], tasks[2], tasks[1], tasks[0]]
    want = []
    for task in seq:
        out = g.run([task])
        want.append({c: (x.m.cpu(), x.e.cpu()) for c, x in out.items()})
    pinned = [dataclasses.replace(task, h_inf={n: mpf.MPF(h.m.pin_memory(), h.e.pin_memory())
                                               for n, h in task.h_inf.items()}) for task in seq]
    got = [{c: (m.clone(), e.clone()) for c, (m, e) in h.items()} for h in g.run_stream([[x] for x in pinned])]
    assert len(got) == len(seq)
    for w, r in zip(want, got):
        assert w.keys() == r.keys()
        for c in w:
            assert torch.equal(w[c][0], r[c][0]) and torch.equal(w[c][1], r[c][1]), c
    assert list(g.run_stream([])) == []


def test_cli_gpu_entry_reads_setup_file(cuda, tmp_path):
    """dropin.gpu, the reference's cli._gpu (same arguments: the cli's tasks, (q4, sign) keys, b3d_setup's file),
    on a setup file holding a group's M matrices and h_inf: the results of run_group on the same numbers, bit for
    bit, in the form the reference's writer consumes (OutputInfo objects with .outputs)"""
    from types import SimpleNamespace
    from blocksvibe_b200 import setup_file as SF
    G, tasks, M, hstr, plan = make_group(nq=2, seed=41, coords=("xt", "xt_radial"))
    L = DI.limbs(G.precision)
    K = (32 * L + 64) // 64 + 2
    with mp.workprec(32 * L + 64):
        mats = {key: [[mp.mpf(x) for x in row] for row in rows] for key, rows in M.items()}
        stasks = []
        for q, t in enumerate(tasks):
            h = {n: [tuple(ent[1:6]) + (mp.mpf(ent[6]),) for ent in hstr[(q, n)]] for n in t.lambda_orders(G.Lambda)}
            stasks.append((t.q4, t.sign, t.pp, h))
    sfile = str(tmp_path / "setup.bin")
    SF.write(sfile, K, mats, stasks)
    cli_tasks = [SimpleNamespace(two_js=list(G.two_js), two_j12=G.two_j12, two_j43=G.two_j43, order=G.order,
                                 Lambda=G.Lambda, tjmax=G.two_j_max, precision=G.precision,
                                 kept_pole_order=G.kept_pole_order, delta_12=G.delta_12, delta_43=G.delta_43,
                                 two_js_internal=list(t.two_js_internal), coordinates=set(t.coordinates),
                                 delta_1_plus_2=t.delta_1_plus_2, q4=list(t.q4), sign=t.sign) for t in tasks]
    timers = []
    got = DI.gpu(cli_tasks, [(tuple(t.q4), t.sign) for t in tasks], sfile, None, timers, device=cuda)
    want = DI.run_group(G, tasks, M, device=cuda)
    assert got.keys() == want.keys()
    for k in want:
        tjs, pp, vals, infos, Smax, NB = got[k]
        assert (tjs, pp, Smax, NB) == (want[k][0], want[k][1], want[k][4], want[k][5])
        assert {c: i.outputs for c, i in infos.items()} == {c: i.outputs for c, i in want[k][3].items()}
        for c in want[k][2]:
            assert np.array_equal(vals[c][0], want[k][2][c][0]) and np.array_equal(vals[c][1], want[k][2][c][1]), c
    assert {name for name, _, _ in timers} >= {".main.gpu.read_setup", ".main.gpu.constants", ".main.gpu.chain"}
