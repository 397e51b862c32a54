"""Serving loop: continuous batching of blocks_3d invocations on one GPU.

Requests (one blocks_3d task each: a group, a task, the group's M matrices) arrive at any time.  Requests that
share an operator (group, pseudo-parities, sign, internal spins, coordinates, Delta_1+2) are batched: one
recursion pass over all their right-hand sides (``dropin.Operator.run_batched``).  Admission is by device
footprint: a batch is formed from the oldest pending requests of one operator while the residue slots,
moments and h_inf of everything in flight fit the HBM budget.  ``workers`` batches run at the same time,
each on its own CUDA stream, so work of different operators overlaps on the device; requests that arrive
while others run join the next batch of their operator.  Every GPU operation is independent per right-hand
side, so a request's result is the same alone and in any mix (tested bit for bit).

    srv = Server(device, budget_bytes=..., workers=2)
    req = srv.submit(group, task, M)        # any thread, any time
    srv.wait(req)                           # -> req.result (the per-task host arrays of dropin.run_group)
    srv.latencies()                         # seconds from arrival to result, per finished request
"""
import threading
import time
from dataclasses import dataclass, field

import torch

from . import dropin as DI


@dataclass
class Request:
    group: DI.Group
    task: DI.Task
    M: object
    arrival: float
    id: int
    footprint: int = 0
    result: object = None
    error: object = None
    done: float = None
    event: threading.Event = field(default_factory=threading.Event)


def operator_key(group, task):
    return (tuple(vars(group).items()), tuple(task.pp), task.sign, tuple(task.two_js_internal),
            tuple(task.coordinates), task.delta_1_plus_2)


class Server:
    def __init__(self, device="cuda", budget_bytes=None, workers=2, max_batch=32, schedule="batched",
                 host_results=True):
        """host_results: copy each result to host arrays (the reference's cli._gpu contract); False keeps it on
        the device as MPF views of the batch output (for the GPU JSON writer, jsonout.SpinWriter)"""
        self.device = torch.device(device)
        self.host_results = host_results
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.5 * free)
        self.budget = budget_bytes
        self.max_batch, self.schedule = max_batch, schedule
        self.lock = threading.Condition()
        self.pending = []                 # Requests in arrival order
        self.in_flight = 0                # bytes admitted and not yet released
        self.peak_in_flight = 0
        self.ops = {}                     # operator key -> dropin.Operator
        self.finished = []
        self.next_id = 0
        self.stop = False
        self.batches = []                 # (operator key, request ids) of every batch run
        self.building = set()
        self._build_stream = torch.cuda.Stream(self.device)
        self.threads = [threading.Thread(target=self._worker, daemon=True) for _ in range(workers)]
        for th in self.threads:
            th.start()

    # ------------------------------------------------------------ client side
    def add_operator(self, op, group, task):
        """register an operator built elsewhere (dropin.Operator) for the requests of (group, task)'s key"""
        with self.lock:
            self.ops[operator_key(group, task)] = op
            self.lock.notify_all()

    def submit(self, group, task, M, arrival=None):
        with self.lock:
            r = Request(group, task, M, time.perf_counter() if arrival is None else arrival, self.next_id)
            self.next_id += 1
            self.pending.append(r)
            self.lock.notify_all()
        return r

    def wait(self, req, timeout=None):
        if not req.event.wait(timeout):
            raise TimeoutError(f"request {req.id} not finished")
        if req.error is not None:
            raise req.error
        return req.result

    def close(self):
        with self.lock:
            self.stop = True
            self.lock.notify_all()
        for th in self.threads:
            th.join()

    def latencies(self):
        return [r.done - r.arrival for r in self.finished]

    # ------------------------------------------------------------ scheduling
    def _ensure_operator(self):
        """build (outside the lock) the operator of the oldest pending request if it does not exist yet"""
        with self.lock:
            if not self.pending:
                return
            head = self.pending[0]
            key = operator_key(head.group, head.task)
            if key in self.ops or key in self.building:
                return
            self.building.add(key)
        try:
            with torch.cuda.stream(self._build_stream):
                op = DI.Operator(head.group, tuple(head.task.pp), head.task.parity, head.M, head.task.two_js_internal,
                                 list(head.task.coordinates), [head.task.delta_1_plus_2], self.device)
                self._build_stream.synchronize()
        except Exception as exc:
            with self.lock:
                self.building.discard(key)
                for r in [r for r in self.pending if operator_key(r.group, r.task) == key]:
                    self.pending.remove(r)
                    r.error, r.done = exc, time.perf_counter()
                    self.finished.append(r)
                    r.event.set()
            return
        with self.lock:
            self.ops[key] = op
            self.building.discard(key)
            self.lock.notify_all()

    def _take_batch(self):
        """under the lock: the oldest pending request's operator, and as many of its pending requests as fit"""
        if not self.pending:
            return None
        head = self.pending[0]
        key = operator_key(head.group, head.task)
        if key not in self.ops:
            return None
        batch, size = [], 0
        for r in self.pending:
            if len(batch) >= self.max_batch:
                break
            if operator_key(r.group, r.task) != key:
                continue
            if r.footprint == 0:
                r.footprint = self._footprint(key, r)
            if batch and self.in_flight + size + r.footprint > self.budget:
                break
            if not batch and self.in_flight + r.footprint > self.budget and self.in_flight > 0:
                return None                                  # wait for memory to be released
            batch.append(r)
            size += r.footprint
        for r in batch:
            self.pending.remove(r)
        self.in_flight += size
        self.peak_in_flight = max(self.peak_in_flight, self.in_flight)
        self.batches.append((key, [r.id for r in batch]))
        return key, batch, size

    def _footprint(self, key, r):
        """device bytes of a request: its residue slots, moments and h_inf, times 1.5 for the temporaries"""
        nrhs = len(r.task.lambda_orders(r.group.Lambda))
        return int(1.5 * self.ops[key].footprint_bytes(nrhs))

    def _worker(self):
        stream = torch.cuda.Stream(self.device)
        while True:
            self._ensure_operator()
            with self.lock:
                got = None
                while got is None:
                    if self.stop and not self.pending:
                        return
                    got = self._take_batch()
                    if got is None:
                        self.lock.wait(0.05)
                        if self.pending and operator_key(self.pending[0].group, self.pending[0].task) not in self.ops:
                            break
                if got is None:
                    continue
                key, batch, size = got
            try:
                with torch.cuda.stream(stream):
                    head = batch[0]
                    op = self.ops[key]
                    ns = head.task.lambda_orders(head.group.Lambda)
                    tasks = [r.task for r in batch]
                    nums = op.run_batched(tasks, ns) if self.schedule == "batched" else op.run_plain(tasks, ns)
                    out = op.apply_outputs(nums, head.task.delta_1_plus_2)
                    if self.host_results:                  # pinned buffers: one asynchronous copy per array
                        host = {}
                        for c, x in out.items():
                            hm = torch.empty(x.m.shape, dtype=torch.int32, pin_memory=True)
                            he = torch.empty(x.e.shape, dtype=torch.int64, pin_memory=True)
                            hm.copy_(x.m, non_blocking=True)
                            he.copy_(x.e, non_blocking=True)
                            host[c] = (hm, he)
                    stream.synchronize()
                now = time.perf_counter()
                d12 = head.task.delta_1_plus_2
                for q, r in enumerate(batch):
                    if self.host_results:
                        r.result = {(c, d12): (m[:, :, :, :, q].numpy(), e[:, :, :, q].numpy()) for c, (m, e) in host.items()}
                    else:
                        r.result = {(c, d12): x[:, :, :, q:q + 1] for c, x in out.items()}
                    r.done = now
            except Exception as exc:                           # surfaced to the waiting client
                for r in batch:
                    r.error = exc
                    r.done = time.perf_counter()
            with self.lock:
                self.in_flight -= size
                self.finished.extend(batch)
                self.lock.notify_all()
            for r in batch:
                r.event.set()


def poisson_arrivals(rate, count, seed=0):
    """arrival offsets (seconds) of a Poisson process of the given rate"""
    import random
    rng = random.Random(seed)
    t, out = 0.0, []
    for _ in range(count):
        t += rng.expovariate(rate)
        out.append(t)
    return out


def replay(server, items, rate, seed=0):
    """submit (group, task, M) items at Poisson arrival times (rate per second, real time); returns the requests
    once all are finished"""
    offsets = poisson_arrivals(rate, len(items), seed)
    t0 = time.perf_counter()
    reqs = []
    for off, (g, t, M) in zip(offsets, items):
        delay = t0 + off - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        reqs.append(server.submit(g, t, M, arrival=t0 + off))
    for r in reqs:
        server.wait(r)
    return reqs, time.perf_counter() - t0


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    return xs[min(len(xs) - 1, int(round(q * (len(xs) - 1))))]
