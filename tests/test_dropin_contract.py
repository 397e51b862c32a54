"""The drop-in boundary on the host (CPU only): the result the drop-in returns is the one the reference's
writer consumes, and b3d_setup's file is read as the reference reads it.

* dropin_write.json holds the spin files the reference's own cli._write -> _write_one -> _rows ->
  b3djson.write_spin produced from results built by dropin.task_results (tests/golden/make_dropin_golden.py);
  here the slot layout is checked and the same files are rebuilt from those results with the host header and
  the oracle's formatter, following the consumer's grouping of output rows.  With the reference at hand
  ($BLOCKSVIBE_REFERENCE), the reference's writer is also run live on them.
* The B3DSETUP reader (setup_file.read, the library's b3d_setup_numbers) against exact values written in the
  layout of the reference's b3d_setup.cxx:15-21 by setup_file.write: numbers rounded once to L limbs as every
  host conversion rounds, M tables placed by plan keys, h_inf in the recursion's layout, malformed files refused.
"""
import os
import sys

import mpmath as mp
import numpy as np
import pytest
import torch

from conftest import GOLDEN, golden
from blocksvibe_b200 import dropin as DI, jsonout as JO, mpf, setup_file as SF
from blocksvibe_b200.plan import Plan
from oracle import jsonfmt as OJ

sys.path.insert(0, GOLDEN)
import dropin_cases as DC                   # noqa: E402
import json_cases as JC                     # noqa: E402


def _results(case):
    vals, outputs, Sm, L = DC.host_values(case)
    d12 = "2.3"
    infos = {(c, d12): DI.OutputInfo(outputs[c]) for c in vals}
    tjs = sorted(case[7])
    per = DI.task_results(tjs, case[4], {(c, d12): v for c, v in vals.items()}, infos, Sm, L, len(DC.Q4S))
    return per, vals, outputs, Sm, L


def _consumer_rows(info, v):
    """the reference consumer's grouping (cli._rows): output rows per first derivative, in output order"""
    rows = {}
    for k, (n, _) in enumerate(info.outputs):
        rows.setdefault(n, []).append(v[k])
    return [rows[n] for n in sorted(rows)]


@pytest.mark.parametrize("ci", range(len(JC.SPIN_CASES)))
def test_results_rebuild_reference_consumer_files(ci):
    g = golden("dropin_write.json")[ci]
    case = JC.SPIN_CASES[ci]
    per, vals, outputs, Sm, L = _results(case)
    pp = case[4]
    for q, (tjs, pp_, res, infos, Smax, NB) in enumerate(per):
        assert pp_ == pp and Smax == Sm and NB == 32 * L - 2
        assert all(hasattr(i, "outputs") for i in infos.values())
        attrs = dict(g["tasks"][q])
        attrs["coordinates"] = set(attrs["coordinates"])
        opts = type("Opts", (), attrs)
        p = JO.digits10(opts.precision)
        for tj in opts.two_js_internal:
            jo = tjs.index(tj)
            structs = [(len(JC.so3(pp[k][0], opts.two_j12, tj)), len(JC.so3(pp[k][1], opts.two_j43, tj)))
                       for k in range(2)]
            coord_rows = []
            for c in [c for c in JO.COORD_ORDER if c in opts.coordinates]:
                m, e = res[(c, opts.delta_1_plus_2)]                     # (L, Jo, 2, S2, outputs, Dmax)
                info = infos[(c, opts.delta_1_plus_2)]

                def num(k, s, o, d):
                    limbs = np.ascontiguousarray(m[:, jo, k, s, o, d]).tobytes()
                    v = int.from_bytes(limbs, "little", signed=True)
                    return (v, int(e[jo, k, s, o, d])) if v else (0, 0)

                def block(k, s):
                    return _consumer_rows(info, [[num(k, s, o, d) for d in range(m.shape[-1])]
                                                 for o in range(len(info.outputs))])
                coord_rows.append([[[block(k, a * Sm + b) for b in range(structs[k][1])] for a in range(structs[k][0])]
                                   for k in range(2)])
            text = JO.header(opts, tj, pp, p) + "  \"derivs\":\n  [\n" + OJ.derivs_body(structs, coord_rows, p) + "\n  ]\n}\n"
            assert text == g["files"][str(q)][str(tj)], (q, tj)


@pytest.mark.skipif(not os.path.isdir(os.environ.get("BLOCKSVIBE_REFERENCE", "") or "/nonexistent"),
                    reason="set BLOCKSVIBE_REFERENCE to the reference's source tree to run its writer live")
def test_reference_writer_consumes_results_live():
    import make_dropin_golden as MG
    import ref_standins
    ref_standins.install(os.environ["BLOCKSVIBE_REFERENCE"])
    from blocksvibe import cli
    for ci, case in enumerate(JC.SPIN_CASES):
        files, _ = MG.consumer_files(cli, case)
        g = golden("dropin_write.json")[ci]["files"]
        assert {str(q): {str(tj): t for tj, t in f.items()} for q, f in files.items()} == g


# ---------------------------------------------------------------- B3DSETUP reader

def _exact_values(rng, n):
    with mp.workprec(2000):
        out = [mp.mpf(0), mp.mpf(1), mp.mpf(-3) / 7, mp.pi * 2 ** 100, -mp.e * mp.mpf(2) ** -300]
        out += [mp.mpf(rng.uniform(-1, 1)) * mp.mpf(2) ** rng.randint(-300, 300) for _ in range(n)]
    return out


def _gmp_truncated(v, K):
    """the value a K-limb GMP mpf holds for v (truncated toward zero)"""
    r = SF._record(v, K)
    if r[0] == 0:
        return mp.mpf(0)
    mag = sum(int(np.int64(x).view(np.uint64)) << (64 * t) for t, x in enumerate(r[2:]))
    return (1 if r[0] > 0 else -1) * mp.ldexp(mp.mpf(mag), 64 * (r[1] - K))


@pytest.mark.parametrize("L,K", [(10, 6), (34, 18), (42, 12), (42, 22)])
def test_setup_numbers_round_once(tmp_path, L, K):
    import random
    vals = _exact_values(random.Random(L * 100 + K), 60)
    path = str(tmp_path / "setup.bin")
    SF.write(path, K, {}, [((2, 2, 0, 0), 1, ((0, 0), (1, 1)), {0: [(0, 1, 2, 0, 0, v) for v in vals]})])
    _, tasks = SF.read(path, L)
    idx, m, e = tasks[0].h[0]
    got = mpf.to_mp(mpf.MPF(torch.from_numpy(m), torch.from_numpy(e)))
    with mp.workprec(4096):
        want = mpf.to_mp(mpf.from_mp([_gmp_truncated(v, K) for v in vals], L))
    assert list(got) == list(want)
    assert idx.tolist() == [[0, 1, 2, 0, 0]] * len(vals)


def test_setup_m_table_and_h_inf_layout(tmp_path):
    import random
    rng = random.Random(7)
    plan = Plan(2, 2, 4, 5, ((0, 1), (1, 0)))
    keys = list(plan.Mkeys)[::3]
    from oracle.sample import RandomMatrices
    mats = {}
    with mp.workprec(400):
        for key in keys:
            r, c = RandomMatrices.shape(key)
            mats[key] = [[mp.mpf(rng.randint(-1000, 1000)) / 64 for _ in range(c)] for _ in range(r)]
        ents = [(s, lev, j, a, b, mp.mpf(rng.randint(1, 99)) / 8) for s in range(2) for lev in (0, 3, 5, 9)
                for j in (0, 2, plan.Jh, plan.Jh + 1) for a in range(2) for b in range(2)]
    path = str(tmp_path / "setup.bin")
    SF.write(path, 8, mats, [((0, 2, 2, 0), -1, ((0, 1), (1, 0)), {1: ents, 3: ents[:5]})])
    M, tasks = SF.read(path, 10)
    T = M.for_plan(plan)
    got = mpf.to_mp(T)
    Sm = plan.Smax
    for key, i in plan.Mkeys.items():
        want = mats.get(key, [])
        for a in range(Sm):
            for b in range(Sm):
                w = want[a][b] if a < len(want) and b < len(want[a]) else 0
                assert got[i, a, b] == w, (key, a, b)
    st = tasks[0]
    assert (st.q4, st.sign, st.pp) == ((0, 2, 2, 0), -1, ((0, 1), (1, 0))) and sorted(st.h) == [1, 3]
    H = mpf.to_mp(st.h_inf(1, 5, plan.Jh, Sm))              # levels <= order and spins < Jh kept
    assert H.shape == (2, 6, plan.Jh, Sm * Sm)
    for s, lev, j, a, b, v in ents:
        if lev <= 5 and j < plan.Jh:
            assert H[s, lev, j, a * Sm + b] == v
    kept = sum(1 for s, lev, j, a, b, v in ents if lev <= 5 and j < plan.Jh)
    assert sum(1 for x in H.reshape(-1) if x) == kept


def test_setup_file_errors(tmp_path):
    path = str(tmp_path / "bad.bin")
    np.array([1, 2, 3], dtype=np.int64).tofile(path)
    with pytest.raises(ValueError, match="not a B3DSETUP"):
        SF.read(path, 10)
    SF.write(path, 4, {}, [((0, 0, 0, 0), 1, ((0, 0), (1, 1)), {0: [(0, 0, 0, 0, 0, mp.mpf(1))]})])
    raw = np.fromfile(path, dtype=np.int64)
    raw[:-1].tofile(path)
    with pytest.raises(ValueError, match="truncated"):
        SF.read(path, 10)
    np.concatenate([raw, [0]]).tofile(path)
    with pytest.raises(ValueError, match="trailing"):
        SF.read(path, 10)
