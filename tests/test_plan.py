"""The vectorised plan builder against golden plans of the reference's builder (recursion_gpu.Plan, which
the reference's tests in turn check against its per-task builder plan_ref.PlanRef): identical scalars,
keys, slot maps and per-level tensors, with and without slot reuse.  Integer work: exact.  CPU only."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from blocksvibe_b200.plan import Plan, cauchy_tables

FIELDS = ("gsrc", "gj", "col", "rowd", "nrow", "cold", "ncol", "t_slot", "t_hrow", "t_L", "t_R", "t_q", "t_qL")


@pytest.fixture(scope="module")
def plans():
    return np.load(os.path.join(GOLDEN, "plan.npz"))


@pytest.mark.parametrize("ci", range(8))
@pytest.mark.parametrize("reuse", [False, True])
def test_plan_matches_reference(plans, ci, reuse):
    c = plans["cases"][ci]
    pp = ((int(c[4]), int(c[5])), (int(c[6]), int(c[7])))
    pl = Plan(int(c[0]), int(c[1]), int(c[2]), int(c[3]), pp, reuse=reuse)
    k = f"c{ci}_r{int(reuse)}_"
    assert [pl.Smax, pl.Jh, pl.nslots, pl.nphys, pl.zero_slot, pl.dmax] == plans[k + "scalars"].tolist()
    mk = [[P[0], P[1], d, tjnn, ppq, tj, i] for (P, d, tjnn, ppq, tj), i in pl.Mkeys.items()]
    assert mk == plans[k + "mkeys"].tolist()
    qk = [[P[0], P[1], tj, sg, i] for (P, tj, sg), i in pl.Qkeys.items()]
    assert qk == plans[k + "qkeys"].tolist()
    assert np.array_equal(np.asarray(pl.LQpairs).reshape(-1, 2), plans[k + "lqpairs"])
    assert np.array_equal(pl.phys, plans[k + "phys"])
    assert [-1 if lev is None else lev["m"] for lev in pl.levels] == plans[k + "levels"].tolist()
    for lev in pl.levels:
        if lev is None:
            continue
        m = lev["m"]
        assert [lev["nb"], lev["Mr"], lev["Kc"]] == plans[k + f"l{m}_dims"].tolist()
        for f in FIELDS:
            assert np.array_equal(np.asarray(lev[f]), plans[k + f"l{m}_{f}"]), (m, f)
        cdiff, _ = cauchy_tables(lev)
        assert np.array_equal(cdiff.astype(np.int64), plans[k + f"l{m}_cdiff"]), m


def test_slot_reuse_shrinks_buffer():
    """recycled physical slots: strictly fewer than logical ones on a recursion deep enough to recycle"""
    a = Plan(4, 2, 8, 12, ((0, 1), (1, 0)), reuse=False)
    b = Plan(4, 2, 8, 12, ((0, 1), (1, 0)), reuse=True)
    assert b.nphys < a.nphys
    # every logical slot written at some level has a physical slot below nphys
    born = b.phys[b.phys >= 0]
    assert born.max() < b.nphys
