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
