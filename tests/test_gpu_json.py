"""GPU JSON output (b3d_format_decimal, b3d_poly_sizes, b3d_emit_text through blocksvibe_b200.jsonout) against
the reference writer's golden output (tests/golden/json_output.json) and the oracle (oracle/jsonfmt.py):
byte-exact numbers, polynomial truncation sizes and complete per-spin files."""
import random
import sys

import numpy as np
import pytest
import torch

from conftest import GOLDEN, golden
from blocksvibe_b200 import jsonout as JO, mpf
from blocksvibe_b200._lib import B3DError
from oracle import jsonfmt as OJ

sys.path.insert(0, GOLDEN)
import json_cases as JC  # noqa: E402

pytestmark = pytest.mark.gpu


def texts(x, p):
    slots, lens = JO.format_numbers(x, p)
    s, ln = slots.cpu().numpy(), lens.cpu().numpy()
    return [bytes(s[i, :ln[i]]).decode() for i in range(len(ln))]


def as_mpf(vals, L, shape, device):
    return mpf.from_ints([v for v, _ in vals], [e for _, e in vals], L, shape, device)


@pytest.mark.parametrize("ci", range(len(JC.NUMBER_CASES)))
def test_numbers_match_reference_writer(cuda, ci):
    g = golden("json_output.json")["numbers"][ci]
    vals = JC.random_numbers(g["L"], g["count"], g["seed"])
    assert texts(as_mpf(vals, g["L"], (len(vals),), cuda), g["p"]) == g["text"]


@pytest.mark.parametrize("L", [10, 18, 34, 42])
def test_numbers_match_oracle_random_and_ties(cuda, L):
    rng = random.Random(L)
    p = JO.digits10(32 * (L - 2))
    NB = 32 * L - 2
    vals = JC.random_numbers(L, 400, 1000 + L)
    vals += [(10 ** p + 5, 0), (10 ** (p - 1) * 10 + 15, -1), (-(2 * 10 ** p + 5), 0), (10 ** p - 1, 0),
             (10 ** p + 4, 0), (10 ** p + 6, 0), ((1 << (NB - 2)) + 1, -(NB - 2))]         # ties and near-ties
    for _ in range(100):                                    # short dyadic values (exact, often tied at p digits)
        vals.append((rng.randint(-10 ** 6, 10 ** 6) or 1, rng.randint(-60, 60)))
    vals = [(v, e) for v, e in vals if abs(v).bit_length() <= NB]
    assert texts(as_mpf(vals, L, (len(vals),), cuda), p) == [OJ.fmt(v, e, p) for v, e in vals]


def test_zero_and_out_of_range(cuda):
    L, p = 10, 77
    x = mpf.from_ints([0, 1, 1], [0, -2000, 0], L, (3,), cuda)       # 2^-2000 ~ 10^-602 < 10^(-2p-1)
    slots, lens = JO.format_numbers(x, p, check=False)
    assert lens.cpu().tolist()[0] == 1 and lens.cpu().tolist()[1] == -1
    with pytest.raises(B3DError):
        JO.check_errors(L, p, cuda)


def test_poly_sizes_match_oracle(cuda):
    L, p, D = 10, 77, 6
    s = JO.eps_shift(p)
    rng = random.Random(5)
    NB = 32 * L - 2
    polys = []
    for t in range(300):
        poly = []
        for d in range(D):
            r = rng.random()
            if r < 0.2:
                poly.append((0, 0))
            else:
                v = rng.getrandbits(NB - 1) | (1 << (NB - 1))
                e = -NB + rng.randint(-40, 40)
                if r < 0.4:
                    e -= s + rng.randint(-3, 3)             # around the truncation threshold
                poly.append((-v if rng.random() < 0.5 else v, e))
        if t % 7 == 0:
            poly = [(0, 0)] * D
        if t % 11 == 0:                                     # exactly at the threshold: kept only if strictly above
            poly = [(1 << (NB - 1), -NB), (1 << (NB - 1), -NB - s)] + [(0, 0)] * (D - 2)
        polys.append(poly)
    flat = [c for poly in polys for c in poly]
    x = as_mpf(flat, L, (len(flat),), cuda)
    _, lens = JO.format_numbers(x, p)
    from blocksvibe_b200 import _lib
    npoly = len(polys)
    poly_num = torch.arange(npoly, dtype=torch.int64, device=cuda) * D
    size = torch.empty(npoly, dtype=torch.int32, device=cuda)
    tlen = torch.empty(npoly, dtype=torch.int64, device=cuda)
    _lib.call("b3d_poly_sizes", L, x.m.data_ptr(), x.e.data_ptr(), x.m.stride(0), poly_num.data_ptr(), npoly, D, s,
              lens.data_ptr(), size.data_ptr(), tlen.data_ptr(), torch.cuda.current_stream(cuda).cuda_stream)
    want = [OJ.poly_size(poly, p) for poly in polys]
    assert size.cpu().tolist() == want
    want_len = [len(OJ.poly_text(poly, p)) for poly in polys]
    assert tlen.cpu().tolist() == want_len


def spin_outputs(case, device):
    opts, outputs, Sm, vals = JC.spin_case(case)
    L = 2 * ((opts.precision + 63) // 64) + 2
    Dmax = case[8]
    outs = {}
    for c, per in vals.items():
        flat = [x for jo in per for k in jo for s in k for o in s for x in o]
        outs[c] = as_mpf(flat, L, (len(per), 2, Sm * Sm, 1, len(outputs[c]), Dmax), device)
    return opts, outputs, Sm, Dmax, outs


@pytest.mark.parametrize("ci", range(len(JC.SPIN_CASES)))
def test_spin_files_match_reference_writer(cuda, ci):
    g = golden("json_output.json")["spins"][ci]
    case = JC.SPIN_CASES[ci]
    opts, outputs, Sm, Dmax, outs = spin_outputs(case, cuda)
    w = JO.SpinWriter(opts, opts.two_js_internal, case[4], outputs, Sm, 1, Dmax, cuda)
    files = w.render(outs, 0)
    assert sorted(files) == sorted(opts.two_js_internal)
    files = {tj: bytes(v) for tj, v in files.items()}
    for tj, text in files.items():
        assert text.decode() == g["files"][str(tj)]
    again = {tj: bytes(v) for tj, v in w.render(outs, 0).items()}     # cached skeleton, same bytes
    assert again == files


def test_spin_file_of_one_task_in_a_batch(cuda):
    """the files of column q of a batched output are those of the task alone"""
    case = JC.SPIN_CASES[0]
    opts, outputs, Sm, Dmax, outs = spin_outputs(case, cuda)
    g = golden("json_output.json")["spins"][0]
    c = "xt"
    x = outs[c]
    other = mpf.random_mpf(tuple(x.shape), x.L, device=cuda)
    both = mpf.cat([other, x], 3)                           # task 1 of a batch of 2
    w = JO.SpinWriter(opts, opts.two_js_internal, case[4], outputs, Sm, 2, Dmax, cuda)
    files = w.render({c: both}, 1)
    for tj, text in files.items():
        assert bytes(text).decode() == g["files"][str(tj)]


def test_write_files(cuda, tmp_path):
    case = JC.SPIN_CASES[1]
    g = golden("json_output.json")["spins"][1]
    opts, outputs, Sm, Dmax, outs = spin_outputs(case, cuda)
    w = JO.SpinWriter(opts, opts.two_js_internal, case[4], outputs, Sm, 1, Dmax, cuda)
    w.write(outs, lambda tj: str(tmp_path / f"spin_{tj}.json"))
    for tj in opts.two_js_internal:
        assert (tmp_path / f"spin_{tj}.json").read_text() == g["files"][str(tj)]


@pytest.mark.parametrize("ci", range(len(JC.SPIN_CASES)))
def test_spinwriter_matches_reference_consumer_of_dropin_results(cuda, ci):
    """the GPU writer on the device form of the drop-in's results (two tasks in one batch) gives the files the
    reference's cli._write wrote from the host form of the same results (tests/golden/dropin_write.json)"""
    from types import SimpleNamespace
    import dropin_cases as DC
    g = golden("dropin_write.json")[ci]
    case = JC.SPIN_CASES[ci]
    vals, outputs, Sm, L = DC.host_values(case)
    outs = {c: mpf.MPF(torch.from_numpy(m).to(cuda), torch.from_numpy(e).to(cuda)) for c, (m, e) in vals.items()}
    Dmax = case[8]
    for q in range(len(DC.Q4S)):
        attrs = dict(g["tasks"][q])
        attrs["coordinates"] = set(attrs["coordinates"])
        opts = SimpleNamespace(**attrs)
        w = JO.SpinWriter(opts, sorted(opts.two_js_internal), case[4], outputs, Sm, len(DC.Q4S), Dmax, cuda)
        files = {tj: bytes(v).decode() for tj, v in w.render(outs, q).items()}
        assert files == {int(tj): t for tj, t in g["files"][str(q)].items()}
