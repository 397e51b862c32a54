"""Bounded CPU samples of the oracle on a benchmark workload, for the CPU baseline of bench.py: the oracle
recursion (fill_residues) run for a fixed time on a random operator of the workload's shape, and the exact
count of multiprecision MACs a full task needs.  Test infrastructure only."""
import random
import time

import mpmath as mp

from . import blocks as B
from .recursion import count_macs, fill_residues


class RandomMatrices:
    """M matrices of any key, random in [-2, 2], created on first use with blocks_3d's shapes"""

    def __init__(self, seed):
        self.rng = random.Random(seed)
        self.cache = {}

    @staticmethod
    def shape(key):
        P, _, tjnn, ppq, tj = key
        rows = len(B.so3((ppq + (1 if P[0] == 3 else 0)) % 2, tjnn, tj))
        cols = len(B.so3(ppq, tjnn, B.child(P, tj)))
        return rows, cols

    def get(self, key, default=None):
        if key not in self.cache:
            r, c = self.shape(key)
            self.cache[key] = [[mp.mpf(self.rng.uniform(-2, 2)) for _ in range(c)] for _ in range(r)]
        return self.cache[key]


class RandomHinf:
    def __init__(self, seed):
        self.rng = random.Random(seed + 1)
        self.cache = {}

    def get(self, key, default=None):
        if key not in self.cache:
            self.cache[key] = mp.mpf(self.rng.uniform(-1, 1))
        return self.cache[key]


class _Shapes:
    def get(self, key, default=None):
        return RandomMatrices.shape(key)


def recursion_macs_per_rhs(tj12, tj43, tj_max, order, pp):
    return count_macs(tj12, tj43, tj_max, order, pp, _Shapes())


def sample(tj12, tj43, tj_max, order, pp, precision_bits, budget_s, seed=0):
    """(MACs done, seconds) of the oracle recursion run for about budget_s seconds"""
    mp.mp.prec = precision_bits
    stats = {}
    t0 = time.perf_counter()
    fill_residues(RandomHinf(seed), RandomMatrices(seed), tj12, tj43, tj_max, order, pp, budget=budget_s, stats=stats)
    return stats["macs"], time.perf_counter() - t0


def _worker(args):
    return sample(*args)


def parallel_sample(tj12, tj43, tj_max, order, pp, precision_bits, budget_s, cores):
    """the sample on `cores` worker processes (spawned), each with its own random operator: total MACs per
    second over all workers"""
    import multiprocessing as mpr
    jobs = [(tj12, tj43, tj_max, order, pp, precision_bits, budget_s, seed) for seed in range(cores)]
    with mpr.get_context("spawn").Pool(cores) as pool:
        out = pool.map(_worker, jobs)
    macs = sum(m for m, _ in out)
    secs = max(s for _, s in out)
    return macs, secs


# ---------------------------------------------------------------- every stage of a task (the CPU baseline's unit)

def _structures(pp, tj12, tj43, tj):
    return sum(len(B.so3(pp[p][0], tj12, tj)) * len(B.so3(pp[p][1], tj43, tj)) for p in range(2))


def task_macs(c):
    """multiprecision MACs of one blocks_3d task of configuration c (keys tj12, tj43, tjmax, order, Lam, kept,
    sign, coords, pp), every stage: per lambda order the recursion (Cauchy and pole steps, as fill_residues
    counts them), the derivative moments (one product by r_c^n and R + 1 weighted sums per residue), c, a, G, the
    polynomial part and the numerator products of each (spin, parity, structure) block; then the write_output
    map on every coefficient.  The count of the algorithm, not of any implementation."""
    tj12, tj43, tjmax, order, pp, Lam = c["tj12"], c["tj43"], c["tjmax"], c["order"], c["pp"], c["Lam"]
    kept = c["kept"] if c["kept"] < order else None
    parity = (1 - c["sign"]) // 2
    radial = all(x.endswith("_radial") for x in c["coords"])
    orders = [parity] if radial else list(range(parity, Lam + 1, 2))
    rec = recursion_macs_per_rhs(tj12, tj43, tjmax, order, pp)
    spins = list(range(tj12 % 2, tjmax + 1, 2))
    per_spin = []
    for tj in spins:
        poles = B.pole_list(tj, tj12, tj43, order)
        appear = sum(sum(1 for m in range(order) if P in B.pole_list(tj, tj12, tj43, order - m)) for P in poles)
        npout = len(B.pole_list(tj, tj12, tj43, kept)) if kept is not None else len(poles)
        per_spin.append((_structures(pp, tj12, tj43, tj), len(poles), appear, npout))
    total = 0
    for n in orders:
        R = Lam - n
        R1 = R + 1
        total += rec
        for S, NP, appear, npout in per_spin:
            total += S * appear * (R1 + 1)                     # moments
            total += S * R1 * (order + 1)                      # c
            total += S * NP * R1 * R1                          # a
            total += S * NP * R * R1                           # G
            total += S * (R1 ** 3 + 2 * R1 * R1)               # polynomial part
            total += S * (npout + R1) * (NP + R1) * R1         # numerators
    Dmax = max(npout for _, _, _, npout in per_spin) + Lam - parity + 1
    nstruct = sum(S for S, _, _, _ in per_spin)
    for coord in c["coords"]:
        O = Lam if coord == "xt" else Lam - parity
        if coord == "xt":
            ins = sum(O - (parity + 2 * i) + 1 for i in range((O - parity) // 2 + 1))
            outs = sum((O - m - parity) // 2 + 1 for m in range(O - parity + 1))
        else:
            ins = outs = O + 1
        total += ins * outs * nstruct * Dmax
    return total


def chain_task_seconds(c, precision_bits, seed=0):
    """a complete task of configuration c through the oracle, one process (recursion, numerators of every block
    with pole shifting, write_output transforms of every coefficient): wall seconds.  Small configurations only
    (it is the measured anchor of the MAC-based CPU baseline)."""
    from . import derivatives as OD, output as OO
    mp.mp.prec = precision_bits
    tj12, tj43, tjmax, order, pp, Lam = c["tj12"], c["tj43"], c["tjmax"], c["order"], c["pp"], c["Lam"]
    kept = c["kept"] if c["kept"] < order else None
    parity = (1 - c["sign"]) // 2
    radial = all(x.endswith("_radial") for x in c["coords"])
    orders = [parity] if radial else list(range(parity, Lam + 1, 2))
    Ms = RandomMatrices(seed)
    t0 = time.perf_counter()
    nums = {}
    for n in orders:
        H = RandomHinf(seed * 100 + n)
        res = fill_residues(H, Ms, tj12, tj43, tjmax, order, pp)
        h = lambda p, m, j, a, b: H.get((p, m, j, a, b))
        r = lambda p, m, j, q, a, b: res.get((p, m, j, q, a, b), mp.mpf(0))
        for tj in range(tj12 % 2, tjmax + 1, 2):
            for p in range(2):
                for a in range(len(B.so3(pp[p][0], tj12, tj))):
                    for b in range(len(B.so3(pp[p][1], tj43, tj))):
                        nums[(n, tj, p, a, b)] = OD.numerators(h, r, tj, p, a, b, order, Lam - n, tj12, tj43, kept)
    for (tj, p, a, b) in {k[1:] for k in nums}:
        D = max(len(poly) for n in orders for poly in nums[(n, tj, p, a, b)])
        for d in range(D):
            table = [[nums[(n, tj, p, a, b)][e][d] if e <= Lam - n and d < len(nums[(n, tj, p, a, b)][e]) else mp.mpf(0)
                      for e in range(Lam - parity + 1)] for n in orders]
            for coord in c["coords"]:
                if coord == "xt":
                    OO.xt(table, Lam, parity, c["d12"])
                else:
                    OO.xt_radial(table[0], Lam, parity, c["d12"])
    return time.perf_counter() - t0
