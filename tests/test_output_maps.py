"""The write_output composite maps built by blocksvibe_b200.output (host, mpmath) against the reference's maps
(output.Output._xt and the radial prefactor product, golden fixtures) and against the oracle's step-by-step
transforms.  CPU only."""
import mpmath as mp
import pytest

from conftest import golden
from blocksvibe_b200 import output as OUT
from oracle import output as OO


@pytest.mark.parametrize("oi", range(5))
def test_maps_match_reference(oi):
    c = golden("output.json")[oi]
    L = 10
    with mp.workprec(32 * L + 128):
        Lam, p, D = c["Lambda"], c["parity"], mp.mpf(c["delta_1_plus_2"])
        W, inputs, outputs = OUT.xt_map(Lam, p, D)
        assert [list(x) for x in inputs] == c["inputs"] and [list(x) for x in outputs] == c["outputs"]
        ref = [[mp.mpf(x) for x in row] for row in c["W_xt"]]
        big = max(abs(x) for row in ref for x in row)
        err = max(abs(W[i, j] - ref[i][j]) for i in range(len(ref)) for j in range(len(ref[0])))
        assert err <= big * mp.mpf(2) ** -270
        T, _, _ = OUT.xt_radial_map(Lam - p, p, D)
        ref = [[mp.mpf(x) for x in row] for row in c["T_radial"]]
        big = max(abs(x) for row in ref for x in row)
        err = max(abs(T[i, j] - ref[i][j]) for i in range(len(ref)) for j in range(len(ref)))
        assert err <= big * mp.mpf(2) ** -270


def test_map_applied_equals_oracle_transforms():
    """W x num == the oracle's step-by-step lambda_lr_to_lrho_lrhob, congruences and zzb_to_xt"""
    import random
    rng = random.Random(3)
    for Lam, p, D in ((8, 0, "1.25"), (7, 1, "0")):
        with mp.workprec(448):
            W, inputs, outputs = OUT.xt_map(Lam, p, mp.mpf(D))
            nL, R = (Lam - p) // 2 + 1, Lam - p
            num = [[mp.mpf(rng.uniform(-1, 1)) if e <= Lam - p - 2 * idx else mp.mpf(0) for e in range(R + 1)]
                   for idx in range(nL)]
            ref = [x for row in OO.xt(num, Lam, p, D) for x in row]
            got = [mp.fsum(W[o, u] * num[i][e] for u, (i, e) in enumerate(inputs)) for o in range(len(outputs))]
            big = max(abs(x) for x in ref)
            assert max(abs(a - b) for a, b in zip(got, ref)) <= big * mp.mpf(2) ** -380
