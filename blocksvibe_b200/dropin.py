"""The drop-in boundary of the hot path: the contract of the reference's ``cli._gpu``
(``blocksvibe/cli.py:375-440``).  A *group* is a set of blocks_3d tasks sharing (j_external, j12, j43,
Delta_12, Delta_43, order, Lambda, j_max, precision, kept_pole_order); its setup data are the M matrices
and, per task, h_infinity for each lambda order (what the reference reads from b3d_setup's B3DSETUP file,
``setup.py:128-180``).  ``run_group`` returns, per task, the write_output results as host limb arrays, the
format ``cli._write_one`` hands to the JSON writer:

    {(q4, sign): (two_js, pp, {(coord, d12): (m (L, Jo, 2, S^2, outputs, Dmax) int32,
                                              e (Jo, 2, S^2, outputs, Dmax) int64)},
                  {(coord, d12): OutputInfo}, Smax, 32 L - 2)}

where OutputInfo.outputs lists the (derivative, derivative) pair of each output row, what the reference's
writer reads (``cli._OutputInfo``, ``cli.py:443-447``, used by ``_write_one`` / ``_rows``, ``cli.py:471-498``).

Two schedules over the same kernels:
  plain    one right-hand side batch per lambda order (all structures of a (pp, sign) subgroup), R = Lambda - n
           per order: the reference's loop (cli.py:415-426);
  batched  every (structure, lambda order) of a subgroup in ONE recursion pass (B = structures x orders),
           moments accumulated once with R = Lambda - parity, numerators finished per lambda order from the
           first R_n + 1 moments (the same sums: the moment of order k only depends on k).

``gpu(tasks, q4s, sfile, mfile, timers)`` is the reference's ``cli._gpu`` itself (same arguments: the cli's
Task objects, their (q4, sign) keys, b3d_setup's file and the cached M file; same result), reading the setup
file with ``setup_file.read``.
"""
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import mpf
from .derivatives import Derivs, resize
from .mpf import MPF
from .output import Output, apply_per_order
from .plan import Plan
from .recursion import Recursion


@dataclass
class Group:
    two_js: tuple                 # external spins (doubled)
    two_j12: int
    two_j43: int
    order: int
    Lambda: int
    two_j_max: int
    precision: int
    kept_pole_order: int
    delta_12: str = "0"
    delta_43: str = "0"


@dataclass
class Task:
    """one blocks_3d invocation of the group: four-point structure q4 (doubled), sign, pseudo-parity types,
    internal spins, coordinates, Delta_1+2, and h_inf per lambda order n: MPF (2, order + 1, Jh, Smax^2)"""
    q4: tuple
    sign: int
    pp: tuple
    two_js_internal: list
    coordinates: tuple
    delta_1_plus_2: str
    h_inf: dict = field(default_factory=dict)

    @property
    def parity(self):
        return (1 - self.sign) // 2

    def lambda_orders(self, Lam):
        radial = all(c.endswith("_radial") for c in self.coordinates)
        return [self.parity] if radial else list(range(self.parity, Lam + 1, 2))


def limbs(precision):
    return mpf.limbs_for_precision(precision)


class OutputInfo:
    """what the JSON writer needs of a write_output map (host only, picklable): its output list"""

    def __init__(self, outputs):
        self.outputs = [tuple(o) for o in outputs]

    def __repr__(self):
        return f"OutputInfo({len(self.outputs)} outputs)"


def task_results(tjs, pp, vals, infos, Smax, L, nq):
    """per task q < nq of a batch: (two_js, pp, {(coord, d12): (m[..., q, :, :], e[..., q, :, :])}, infos, Smax,
    32 L - 2) from host arrays vals[(coord, d12)] = (m (L, Jo, 2, S^2, nq, outputs, Dmax), e (Jo, 2, S^2, nq,
    outputs, Dmax))"""
    return [(tjs, pp, {k: (m[:, :, :, :, q], e[:, :, :, q]) for k, (m, e) in vals.items()}, infos, Smax, 32 * L - 2)
            for q in range(nq)]


class Operator:
    """Plan + recursion constants + derivative constants + write_output maps of one (pp, sign) subgroup,
    built once and reused for every batch (the reference rebuilds them per subgroup: cli.py:401-406)."""

    def __init__(self, group, pp, parity, M, two_js, coords, d12s, device="cuda"):
        self.group, self.pp, self.parity = group, pp, parity
        self.L = limbs(group.precision)
        self.plan = Plan(group.two_j12, group.two_j43, group.two_j_max, group.order, pp, reuse=True)
        if hasattr(M, "for_plan"):                      # a setup file's M table
            M = M.for_plan(self.plan, device)
        self.rec = Recursion(self.plan, M, self.L, device=device)
        self.der = Derivs(self.plan, group.Lambda - parity, self.L, two_js=two_js,
                          kept_pole_order=group.kept_pole_order, device=device)
        self.outs = {(c, d): Output(c, group.Lambda, parity, d, self.der.Ld, device) for c in coords for d in d12s}
        self.device = torch.device(device)

    def footprint_bytes(self, B):
        return self.rec.footprint_bytes(B) + self.der.footprint_bytes(B) + \
            (4 * self.L + 8) * 2 * (self.group.order + 1) * self.plan.Jh * self.plan.Smax ** 2 * B

    def hinf_batch(self, tasks, ns):
        """h_inf MPF (2, order + 1, Jh, S^2, len(tasks) * len(ns)), rhs index = task * len(ns) + order index"""
        cols = [t.h_inf[n] for t in tasks for n in ns]
        m = torch.stack([c.m for c in cols], -1).to(self.device, non_blocking=True)
        e = torch.stack([c.e for c in cols], -1).to(self.device, non_blocking=True)
        return MPF(m, e)

    def run_plain(self, tasks, ns):
        """reference schedule: per lambda order one recursion over the structures; returns per-order numerators"""
        G = self.group
        nums = []
        for n in ns:
            d = self.der.for_order(G.Lambda - n)
            h = self.hinf_batch(tasks, [n])
            d.start(len(tasks))
            self.rec.run(h, hook=d.accumulate)
            nums.append(d.finish(h))
        return nums

    def run_batched(self, tasks, ns):
        """one recursion pass over every (structure, lambda order); numerators per order from the shared moments"""
        return self.run_batched_h(self.hinf_batch(tasks, ns), len(tasks), ns)

    def run_batched_h(self, h, nq, ns):
        """run_batched on h_inf already on the device: MPF (2, order + 1, Jh, S^2, nq * len(ns))"""
        G = self.group
        no = len(ns)
        d = self.der.for_order(self.der.R)                 # own accumulators: concurrent batches may share self
        d.start(nq * no)
        self.rec.run(h, hook=d.accumulate)
        d.flush()
        S2 = self.plan.Smax ** 2
        mom = d.mom.reshape(d.mom.shape[0], d.R + 1, S2, nq, no)
        nums = []
        for idx, n in enumerate(ns):
            dn = d.for_order(G.Lambda - n)
            R1 = dn.R + 1
            dn.B, dn.N = nq, S2 * nq
            dn.mom = MPF(mom.m[:, :, :R1, :, :, idx], mom.e[:, :R1, :, :, idx]).contiguous().reshape(-1, R1, S2 * nq)
            hn = MPF(h.m.reshape(*h.m.shape[:-1], nq, no)[..., idx], h.e.reshape(*h.e.shape[:-1], nq, no)[..., idx]).contiguous()
            nums.append(dn.finish(hn))
        return nums

    def apply_outputs(self, nums, d12):
        """write_output of the numerators (derivative limbs), rounded to the task's L limbs"""
        return {c: resize(apply_per_order(o, nums), self.L) for (c, dd), o in self.outs.items() if dd == d12}

    def to_host(self, outs):
        """device results -> host limb arrays through reusable pinned buffers (one D2H copy per array)"""
        host = {}
        for c, r in outs.items():
            key = (c, tuple(r.m.shape))
            buf = getattr(self, "_pinned", {}).get(key)
            if buf is None:
                buf = (torch.empty(r.m.shape, dtype=torch.int32, pin_memory=True),
                       torch.empty(r.e.shape, dtype=torch.int64, pin_memory=True))
                self._pinned = getattr(self, "_pinned", {})
                self._pinned[key] = buf
            buf[0].copy_(r.m, non_blocking=True)
            buf[1].copy_(r.e, non_blocking=True)
            host[c] = buf
        torch.cuda.current_stream(self.device).synchronize()
        return host


class GraphStep:
    """The batched step of nq tasks (every lambda order: recursion, moments, numerators, write_output maps)
    captured once as a CUDA graph and replayed per batch: no host work between the ~10^3 launches of a step.
    h: the static device input (2, order + 1, Jh, S^2, nq * len(ns)); out: the static device results."""

    def __init__(self, op, nq, ns, d12):
        self.op, self.nq, self.ns, self.d12 = op, nq, list(ns), d12
        G, pl, L, dev = op.group, op.plan, op.L, op.device
        shape = (2, G.order + 1, pl.Jh, pl.Smax ** 2, nq * len(ns))
        self.h = mpf.zeros(shape, L, dev)
        self.stage = mpf.zeros((nq * len(ns),) + shape[:-1], L, dev)
        op.apply_outputs(op.run_batched_h(self.h, nq, ns), d12)        # warm-up: builds every cached table
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = op.apply_outputs(op.run_batched_h(self.h, nq, ns), d12)
        torch.cuda.synchronize(dev)

    def load(self, tasks):
        """copy the tasks' h_inf (host or device MPFs, one per lambda order) into the static input"""
        k = 0
        for t in tasks:
            for n in self.ns:
                self.stage.m[:, k].copy_(t.h_inf[n].m, non_blocking=True)
                self.stage.e[k].copy_(t.h_inf[n].e, non_blocking=True)
                k += 1
        self.h.m.copy_(self.stage.m.permute(0, 2, 3, 4, 5, 1))
        self.h.e.copy_(self.stage.e.permute(1, 2, 3, 4, 0))

    def run(self, tasks=None):
        if tasks is not None:
            self.load(tasks)
        self.graph.replay()
        return self.out

    def _pipeline_buffers(self):
        dev, L = self.op.device, self.op.L
        copy = torch.cuda.Stream(dev)
        stage = [self.stage, mpf.zeros(tuple(self.stage.shape), L, dev)]
        outd = [{c: (torch.empty_like(x.m), torch.empty_like(x.e)) for c, x in self.out.items()} for _ in range(2)]
        host = [{c: (torch.empty(x.m.shape, dtype=torch.int32, pin_memory=True),
                     torch.empty(x.e.shape, dtype=torch.int64, pin_memory=True)) for c, x in self.out.items()}
                for _ in range(2)]
        in_ready = [torch.cuda.Event() for _ in range(2)]      # inputs of the slot are on the device
        in_free = [torch.cuda.Event() for _ in range(2)]       # the step has taken them into the static input
        out_ready = [torch.cuda.Event() for _ in range(2)]     # results copied out of the static output
        host_ready = [torch.cuda.Event() for _ in range(2)]    # results on the host; the device copy is free
        return copy, stage, outd, host, in_ready, in_free, out_ready, host_ready

    def run_stream(self, batches):
        """Pipelined replays.  For each list of host tasks (h_inf in pinned memory) taken from `batches`, yields
        the results as pinned host arrays {coordinate: (m, e)}, in order; an item stays valid until the next
        one is requested.  A copy stream moves batch i + 1's inputs in and batch i - 1's results out while
        batch i's graph runs, so the host transfers overlap the step; the step's stream itself only adds two
        device-to-device copies (inputs into the static buffer, results out of it).  Staging buffers, device
        result copies and host buffers are double-buffered, every reuse ordered by an event; they are allocated on
        the first call and kept for the next ones."""
        dev = self.op.device
        main = torch.cuda.current_stream(dev)
        if getattr(self, "_pipe", None) is None:               # built once, reused by every call
            self._pipe = self._pipeline_buffers()
        copy, stage, outd, host, in_ready, in_free, out_ready, host_ready = self._pipe

        def bring_in(j, tasks):
            with torch.cuda.stream(copy):
                copy.wait_event(in_free[j])
                k = 0
                for t in tasks:
                    for n in self.ns:
                        stage[j].m[:, k].copy_(t.h_inf[n].m, non_blocking=True)
                        stage[j].e[k].copy_(t.h_inf[n].e, non_blocking=True)
                        k += 1
                in_ready[j].record(copy)

        it = iter(batches)
        nxt = next(it, None)
        if nxt is None:
            return
        bring_in(0, nxt)
        prev, i = None, 0
        while nxt is not None:
            j = i % 2
            nxt = next(it, None)
            if nxt is not None:
                bring_in(1 - j, nxt)
            main.wait_event(in_ready[j])
            self.h.m.copy_(stage[j].m.permute(0, 2, 3, 4, 5, 1))
            self.h.e.copy_(stage[j].e.permute(1, 2, 3, 4, 0))
            in_free[j].record(main)
            self.graph.replay()
            main.wait_event(host_ready[j])
            for c, x in self.out.items():
                outd[j][c][0].copy_(x.m)
                outd[j][c][1].copy_(x.e)
            out_ready[j].record(main)
            with torch.cuda.stream(copy):
                copy.wait_event(out_ready[j])
                for c in self.out:
                    host[j][c][0].copy_(outd[j][c][0], non_blocking=True)
                    host[j][c][1].copy_(outd[j][c][1], non_blocking=True)
                host_ready[j].record(copy)
            if prev is not None:
                host_ready[prev].synchronize()
                yield host[prev]
            prev, i = j, i + 1
        host_ready[prev].synchronize()
        yield host[prev]


def _d12s(task):
    """a task's Delta_1+2 values (one string, or several for a structure written at more than one)"""
    d = task.delta_1_plus_2
    return list(d) if isinstance(d, (list, tuple)) else [d]


def run_group(group, tasks, M, device="cuda", schedule="batched", max_rhs=None, timers=None):
    """All tasks of one group on the GPU.  M: matrices for the plan's keys (dict of decimal strings, a setup
    file's MTable, or an MPF table in plan.Mkeys order; per pseudo-parity subgroup: {pp: M}).  Returns the
    per-task host results described in the module docstring; timers (a list) receives blocks_3d-style
    (name, seconds, count) entries as the reference's _gpu records them."""
    sub = {}
    for t in tasks:
        sub.setdefault((tuple(t.pp), t.sign), []).append(t)
    results = {}
    tick = lambda: (torch.cuda.synchronize(device), time.time())[1]
    for (pp, sign), ts in sub.items():
        parity = (1 - sign) // 2
        ns = sorted(set().union(*[t.lambda_orders(group.Lambda) for t in ts]))
        tjs = sorted(set().union(*[t.two_js_internal for t in ts]))
        coords = [c for c in ("xt", "xt_radial") if any(c in t.coordinates for t in ts)]
        d12s = sorted({d for t in ts for d in _d12s(t)})
        t0 = tick()
        op = Operator(group, pp, parity, M[pp] if isinstance(M, dict) and pp in M else M, tjs, coords, d12s, device)
        infos = {k: OutputInfo(o.outputs) for k, o in op.outs.items()}
        t1 = tick()
        bmax = max_rhs or len(ts)
        chain = out = 0.0
        for c0 in range(0, len(ts), bmax):
            ch = ts[c0:c0 + bmax]
            s0 = tick()
            nums = op.run_batched(ch, ns) if schedule == "batched" else op.run_plain(ch, ns)
            s1 = tick()
            vals = {}
            for d12 in d12s:
                for c, (m, e) in op.to_host(op.apply_outputs(nums, d12)).items():   # (Jo, 2, S2, nq, outputs, Dmax)
                    vals[(c, d12)] = (m.numpy().copy(), e.numpy().copy())
            for t, r in zip(ch, task_results(tjs, pp, vals, infos, op.plan.Smax, op.L, len(ch))):
                results[(tuple(t.q4), t.sign)] = r
            chain += s1 - s0
            out += tick() - s1
        if timers is not None:
            nb = -(-len(ts) // bmax)
            timers += [(".main.gpu.constants", t1 - t0, 1), (".main.gpu.chain", chain, len(ns) * nb),
                       (".main.gpu.write_output", out, 1)]
    return results


def gpu(tasks, q4s, sfile, mfile, timers, device="cuda", schedule="batched"):
    """The reference's ``cli._gpu`` (``cli.py:375-440``): tasks are the cli's Task objects of one group (two_js,
    two_j12, two_j43, order, Lambda, tjmax, precision, kept_pole_order, delta_12, delta_43, two_js_internal,
    coordinates, delta_1_plus_2, q4, sign), q4s their (q4, sign) keys, sfile b3d_setup's file and mfile the
    cached M matrices (or None).  Returns {(q4, sign): (two_js, pp, {(coord, d12): (m, e)}, {(coord, d12):
    OutputInfo}, Smax, 32 L - 2)}, the dict cli._write consumes."""
    from . import setup_file
    T = tasks[0]
    L = limbs(T.precision)
    t0 = time.time()
    M, stasks = setup_file.read(sfile, L, m_path=mfile)
    by_q4 = {(st.q4, st.sign): st for st in stasks}
    timers.append((".main.gpu.read_setup", time.time() - t0, 1))
    group = Group(tuple(T.two_js), T.two_j12, T.two_j43, T.order, T.Lambda, T.tjmax, T.precision,
                  min(T.kept_pole_order, T.order), str(T.delta_12), str(T.delta_43))
    wanted = {(tuple(q), s) for q, s in q4s}
    runs = []
    for t in tasks:
        key = (tuple(t.q4), t.sign)
        if key not in wanted or key not in by_q4 or any(key == (tuple(r.q4), r.sign) for r in runs):
            continue
        st = by_q4[key]
        run = Task(key[0], t.sign, st.pp, list(t.two_js_internal), tuple(sorted(t.coordinates)), t.delta_1_plus_2)
        runs.append(run)
    # the subgroup's union of spins, coordinates and Delta_1+2 (as the reference computes it per subgroup)
    for r in runs:
        same = [t for t in tasks if t.sign == r.sign and by_q4.get((tuple(t.q4), t.sign)) is not None
                and by_q4[(tuple(t.q4), t.sign)].pp == r.pp]
        r.two_js_internal = sorted(set().union(*[t.two_js_internal for t in same]))
        r.coordinates = tuple(c for c in ("xt", "xt_radial") if any(c in t.coordinates for t in same))
        d12s = sorted({t.delta_1_plus_2 for t in same})
        r.delta_1_plus_2 = d12s[0] if len(d12s) == 1 else tuple(d12s)
    plans = {}
    for r in runs:
        key = r.pp
        if key not in plans:
            plans[key] = Plan(group.two_j12, group.two_j43, group.two_j_max, group.order, r.pp)
        pl = plans[key]
        for n in r.lambda_orders(group.Lambda):
            r.h_inf[n] = by_q4[(tuple(r.q4), r.sign)].h_inf(n, group.order, pl.Jh, pl.Smax)
    return run_group(group, runs, M, device=device, schedule=schedule, timers=timers)
