"""Synthetic blocks_3d workloads of the benchmark configurations (random operators: the cost of the path does
not depend on the values, as the reference's own benchmarks assume, recursion_gpu.py:82-88).

  cfg1  (0,0,0,0), 2j12 = 2j43 = 0, spins 0-6, Lambda 5, order 10, kept 6, 256 bits, one xt task
  cfg2  j = (2,2,2,2), 2j12 = 2j43 = 8, spins 0-22, Lambda 11, order 40, kept 20, 1024 bits, one xt task
  cfg5  j = (2,2,2,2), 2j12 = 2j43 = 8, spins 0-40, Lambda 27, order 80, kept 40, 1280 bits, xt_radial
  set644 the 644-task stress-tensor-like set (uneven spins, Lambda in {7, 11, 15}, 768-1024 bits)
"""
import random

import torch

from . import dropin as DI, mpf
from .plan import Plan

PP_SETS = (((0, 0), (1, 1)), ((0, 1), (1, 0)), ((0, 1), (1, 1)), ((1, 0), (0, 1)))

CONFIGS = {
    "cfg1": dict(two_js=(0, 0, 0, 0), tj12=0, tj43=0, tjmax=12, Lam=5, order=10, kept=6, precision=256,
                 coords=("xt",), d12="0", pp=((0, 0), (1, 1)), sign=1),
    "cfg2": dict(two_js=(4, 4, 4, 4), tj12=8, tj43=8, tjmax=44, Lam=11, order=40, kept=20, precision=1024,
                 coords=("xt",), d12="6", pp=((0, 0), (1, 1)), sign=1),
    "cfg2_44": dict(two_js=(4, 4, 4, 4), tj12=4, tj43=4, tjmax=44, Lam=11, order=40, kept=20, precision=1024,
                    coords=("xt",), d12="6", pp=((0, 0), (1, 1)), sign=1),
    "cfg5": dict(two_js=(4, 4, 4, 4), tj12=8, tj43=8, tjmax=80, Lam=27, order=80, kept=40, precision=1280,
                 coords=("xt_radial",), d12="6", pp=((0, 0), (1, 1)), sign=1),
}


def group_of(c):
    return DI.Group(c["two_js"], c["tj12"], c["tj43"], c["order"], c["Lam"], c["tjmax"], c["precision"], c["kept"])


def make_tasks(c, nq=1, seed=0, host=True):
    """nq tasks of config c with random h_inf (host tensors, pinned when CUDA is available)"""
    G = group_of(c)
    L = DI.limbs(G.precision)
    plan = Plan(G.two_j12, G.two_j43, G.two_j_max, G.order, c["pp"])
    g = torch.Generator().manual_seed(seed)
    tasks = []
    for q in range(nq):
        t = DI.Task((q, 0, 0, 0), c["sign"], c["pp"], list(range(c["tj12"] % 2, c["tjmax"] + 1, 2)), c["coords"], c["d12"])
        for n in t.lambda_orders(G.Lambda):
            h = mpf.random_mpf((2, G.order + 1, plan.Jh, plan.Smax ** 2), L, spread=2, generator=g)
            if host and torch.cuda.is_available():
                h = mpf.MPF(h.m.pin_memory(), h.e.pin_memory())
            t.h_inf[n] = h
        tasks.append(t)
    return G, tasks


def task_set_644(seed=644):
    """the 644-task synthetic set: (group spec dict, task count) entries.  External spin sets uniform over the
    four stress-tensor-like ones, j12 / j43 among the so3-allowed values, spin upper bound uniform in 4..30,
    Lambda in {7, 11, 15}, order 2 Lambda + 18, kept Lambda + 9, precision in {768, 896, 1024}, xt or xt_radial."""
    rng = random.Random(seed)
    ext = [(0, 0, 0, 0), (4, 4, 4, 4), (1, 1, 1, 1), (4, 0, 0, 4)]
    out = []
    while sum(n for _, n in out) < 644:
        tj = rng.choice(ext)
        j12 = list(range(abs(tj[0] - tj[1]), tj[0] + tj[1] + 1, 2))     # doubled j12 allowed by the external pair
        j43 = list(range(abs(tj[3] - tj[2]), tj[3] + tj[2] + 1, 2))
        Lam = rng.choice((7, 11, 15))
        spin_top = rng.randint(4, 30)
        tj12, tj43 = rng.choice(j12), rng.choice(j43)
        c = dict(two_js=tj, tj12=tj12, tj43=tj43, tjmax=2 * spin_top + tj12 % 2, Lam=Lam,
                 order=2 * Lam + 18, kept=Lam + 9, precision=rng.choice((768, 896, 1024)),
                 coords=(rng.choice(("xt", "xt_radial")),), d12=f"{rng.uniform(-1, 1):.30f}",
                 pp=rng.choice(PP_SETS) if tj12 and tj43 else PP_SETS[0], sign=rng.choice((1, -1)))
        n = min(rng.randint(1, 22), 644 - sum(k for _, k in out))
        out.append((c, n))
    return out


def make_device_tasks(c, nq, device, seed=0):
    """nq tasks of config c with random h_inf generated on the device (large task sets)"""
    G = group_of(c)
    L = DI.limbs(G.precision)
    plan = Plan(G.two_j12, G.two_j43, G.two_j_max, G.order, c["pp"])
    gen = torch.Generator(device=device).manual_seed(seed)
    tasks = []
    for q in range(nq):
        t = DI.Task((q, 0, 0, 0), c["sign"], c["pp"], list(range(c["tj12"] % 2, c["tjmax"] + 1, 2)), c["coords"], c["d12"])
        for n in t.lambda_orders(G.Lambda):
            t.h_inf[n] = random_mpf_device((2, G.order + 1, plan.Jh, plan.Smax ** 2), L, device, gen)
        tasks.append(t)
    return G, tasks


def random_mpf_device(shape, L, device, gen, spread=2):
    """random normalised values drawn on the device (|x| in about [2^-spread, 2^spread])"""
    from math import prod
    n = prod(shape)
    NB = mpf.nbits(L)
    m = torch.randint(-2 ** 31, 2 ** 31 - 1, (L, n), dtype=torch.int32, device=device, generator=gen)
    top = NB - 32 * (L - 1)
    hi = (m[L - 1].to(torch.int64) & ((1 << (top - 1)) - 1)) | (1 << (top - 1))    # positive, exactly NB bits
    m[L - 1] = hi.to(torch.int32)
    e = torch.randint(-spread, spread + 1, (n,), device=device, generator=gen) - NB
    return mpf.MPF(m.reshape((L,) + tuple(shape)), e.reshape(shape))
