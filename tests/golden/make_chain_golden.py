"""Writes the full-size chain fixtures tests/golden/chain_<case>.json.gz: the oracle (oracle/, the CPU
restatement pinned against the reference's own code by test_oracle_golden.py) run offline on the inputs of
chain_cases.py, on all host cores: the recursion level by level (each level's spins split over worker
processes forked with the residues of the levels below), then the numerators of sampled blocks (and their
xt_radial outputs) in parallel.

    python tests/golden/make_chain_golden.py [--procs N] [case ...]

Each fixture holds sampled residue blocks (parity, level, spin index, pole index: all S_L x S_R entries) and
sampled output blocks (spin, parity, structure a, b: numerator polynomials for every e <= R, or the xt_radial
outputs), every block as integers relative to its largest entry with 32 L bits.  Minutes of CPU time: cfg2_n0
is about 1.9e8 multiprecision MACs of recursion, cfg5_radial about 6.8e8.
"""
import argparse
import gzip
import json
import multiprocessing
import os
import random
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import mpmath as mp                                     # noqa: E402

import chain_cases as CC                                # noqa: E402
from oracle import blocks as OB, derivatives as OD, output as OO, recursion as OR   # noqa: E402


class Matrices:
    """M of a case: key -> matrix of exact mpmath numbers, built on first use"""

    def __init__(self, seed):
        self.seed, self.cache = seed, {}

    def get(self, key, default=None):
        if key not in self.cache:
            r, c = CC.m_shape(key)
            self.cache[key] = [[mp.ldexp(mp.mpf(i), e) for i, e in (CC.m_entry(self.seed, key, a, b) for b in range(c))]
                               for a in range(r)]
        return self.cache[key]


class Hinf:
    """h_inf of a case: (src, m, jh, a, b) -> exact mpmath number, zero outside the GPU tensor's range
    (m <= order, jh < Jh: the spins of level 0 at order + 1)"""

    def __init__(self, c):
        self.seed, self.cache = c["seed"], {}
        self.order, self.Jh = c["order"], len(OB.spins(0, c["order"] + 1, c["tj12"], c["tjmax"]))

    def get(self, key, default=None):
        if key not in self.cache:
            src, m, jh, a, b = key
            if m > self.order or jh >= self.Jh:
                self.cache[key] = mp.mpf(0)
            else:
                i, e = CC.h_entry(self.seed, *key)
                self.cache[key] = mp.ldexp(mp.mpf(i), e)
        return self.cache[key]


_STATE = {}


def _level_part(jsel):
    s = _STATE
    c = s["case"]
    with mp.workprec(32 * c["L"] + 64):
        out, _, _ = OR.fill_level(s["h"], s["M"], s["res"], s["m"], c["tj12"], c["tj43"], c["tjmax"], c["order"],
                                  c["pp"], jsel=set(jsel))
    return out


def recursion(c, procs):
    h, M = Hinf(c), Matrices(c["seed"])
    res = {}
    ctx = multiprocessing.get_context("fork")
    for m in range(c["order"]):
        nsp = len(OB.spins(m, c["order"], c["tj12"], c["tjmax"]))
        nchunk = min(nsp, 4 * procs)
        chunks = [list(range(i, nsp, nchunk)) for i in range(nchunk)]
        _STATE.update(case=c, h=h, M=M, res=res, m=m)
        with ctx.Pool(procs) as pool:
            for part in pool.imap_unordered(_level_part, chunks):
                res.update(part)
        print(f"  level {m}: {len(res)} residues", flush=True)
    return h, res


def _block_outputs(blk):
    s = _STATE
    c = s["case"]
    tj, p, a, b = blk
    R = c["Lam"] - c["n"]
    with mp.workprec(32 * c["L"] + 64):
        hh = lambda pp_, m, j, aa, bb: s["h"].get((pp_, m, j, aa, bb))
        rr = lambda pp_, m, j, q, aa, bb: s["res"].get((pp_, m, j, q, aa, bb), mp.mpf(0))
        polys = OD.numerators(hh, rr, tj, p, a, b, c["order"], R, c["tj12"], c["tj43"], c["kept"])
        if c["coord"] != "xt_radial":
            return blk, [CC.encode(poly, 32 * c["L"]) for poly in polys]
        D = max(len(x) for x in polys)
        rows = []
        for dcoef in range(D):
            col = [polys[e][dcoef] if dcoef < len(polys[e]) else mp.mpf(0) for e in range(R + 1)]
            rows.append(OO.xt_radial(col, c["Lam"], c["n"] % 2, c["d12"]))
        # per output derivative o: its polynomial in x (coefficients d), relative to its largest coefficient
        return blk, [CC.encode([rows[d][o] for d in range(D)], 32 * c["L"]) for o in range(len(rows[0]))]


def sample_blocks(c, res, rng):
    keys = sorted({k[:4] for k in res})
    res_keys = sorted(rng.sample(keys, min(c["res_blocks"], len(keys))))
    out_blocks = []
    spins = list(range(c["tj12"] % 2, c["tjmax"] + 1, 2))
    want = [spins[round(i * (len(spins) - 1) / max(c["num_blocks"] - 1, 1))] for i in range(c["num_blocks"])]
    for tj in want:
        p = rng.randrange(2)
        na, nb = len(CC.so3(c["pp"][p][0], c["tj12"], tj)), len(CC.so3(c["pp"][p][1], c["tj43"], tj))
        if na and nb:
            out_blocks.append((tj, p, rng.randrange(na), rng.randrange(nb)))
    return res_keys, out_blocks


def make(name, procs):
    c = dict(CC.CASES[name])
    t0 = time.time()
    print(f"{name}: recursion", flush=True)
    h, res = recursion(c, procs)
    t1 = time.time()
    rng = random.Random(c["seed"])
    res_keys, out_blocks = sample_blocks(c, res, rng)
    bits = 32 * c["L"]
    residues = []
    with mp.workprec(32 * c["L"] + 64):
        for (p, m, j, q) in res_keys:
            ents = sorted((k[4], k[5]) for k in res if k[:4] == (p, m, j, q))
            E, hx = CC.encode([res[(p, m, j, q, a, b)] for a, b in ents], bits)
            residues.append([p, m, j, q, [list(x) for x in ents], E, hx])
    print(f"{name}: outputs of {len(out_blocks)} blocks", flush=True)
    _STATE.update(case=c, h=h, res=res)
    with multiprocessing.get_context("fork").Pool(procs) as pool:
        outs = pool.map(_block_outputs, out_blocks)
    doc = {"case": name, "bits": bits, "residues": residues,
           "outputs": [[list(blk), val] for blk, val in outs],
           "seconds": {"recursion": round(t1 - t0, 1), "total": round(time.time() - t0, 1)}}
    path = os.path.join(HERE, f"chain_{name}.json.gz")
    with gzip.open(path, "wt") as f:
        json.dump(doc, f)
    print(f"{name}: wrote {path} ({os.path.getsize(path)} bytes) in {time.time() - t0:.0f} s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("cases", nargs="*", default=list(CC.CASES))
    a = ap.parse_args()
    for name in a.cases:
        make(name, a.procs)


if __name__ == "__main__":
    main()
