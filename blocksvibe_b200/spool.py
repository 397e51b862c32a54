"""Spool front end: concurrent blocks_3d invocations (hyperion runs one process per four-point structure) fed
into one continuous-batching serving loop on the GPU.  Replaces the reference's ``cli.spool_run``
(``blocksvibe/cli.py:569-637``), which lets one process per group wait for a quiet window (3 s by default) and
then runs the pending invocations as one batch; here a task is admitted the moment it is claimed, while
earlier ones are on the GPU, and tasks of every group share the one loop (its admission is by HBM footprint,
``serve.Server``).

Protocol (one spool directory per GPU; every file is written atomically, by rename):

    <tid>.task               an invocation waiting: JSON {"argv0": ..., "argv": [...]}
    <tid>.claimed.<pid>      claimed by the serving process <pid>
    <tid>.done               its exit status, written by the serving process
    server.lock              flock held by the serving process for as long as it serves

Every invocation writes its .task and waits for its .done.  While no process holds server.lock, the first
invocation to take it becomes the serving process: it claims every .task (its own included) as it appears,
hands each to the backend, writes the .done files as results come back, and releases the lock after ``idle``
seconds without work.  An invocation whose task was claimed by a serving process that died puts the task
back (renames it to .task), and the next serving process runs it (the reference's recovery, cli.py:596-604).

The backend does the work: ``submit(tid, spec)`` starts a task (must not block for long) and ``poll()``
returns the finished ones as (tid, exit status).  ``ServingBackend`` runs tasks through ``serve.Server``; tests
use a host-only fake.
"""
import errno
import fcntl
import json
import os
import threading
import time
import uuid


def _atomic_write(path, text):
    tmp = f"{path}.tmp{os.getpid()}.{threading.get_ident()}"
    with open(tmp, "w") as f:
        f.write(text)
    os.replace(tmp, path)


def pid_alive(pid):
    try:
        os.kill(pid, 0)
    except OSError as e:
        return e.errno == errno.EPERM
    return True


class SpoolServer:
    """The serving side: claims tasks from the spool directory and drives the backend until idle."""

    def __init__(self, spool_dir, backend, idle=2.0, poll=0.02):
        self.dir, self.backend, self.idle, self.poll = spool_dir, backend, idle, poll
        self.pid = os.getpid()
        self.claimed = []                  # tids in claim order (for tests and logs)

    def _claim(self):
        got = []
        for f in sorted(os.listdir(self.dir)):
            if not f.endswith(".task"):
                continue
            tid = f[:-5]
            dst = os.path.join(self.dir, f"{tid}.claimed.{self.pid}")
            try:
                os.rename(os.path.join(self.dir, f), dst)
            except OSError:                # taken back or claimed meanwhile
                continue
            try:
                with open(dst) as fh:
                    spec = json.load(fh)
            except (OSError, ValueError):
                self._finish(tid, 2)       # unreadable task file: fail that invocation only
                continue
            got.append((tid, spec))
        return got

    def _finish(self, tid, status):
        _atomic_write(os.path.join(self.dir, f"{tid}.done"), str(int(status)))
        try:
            os.remove(os.path.join(self.dir, f"{tid}.claimed.{self.pid}"))
        except OSError:
            pass

    def serve(self):
        """run until no task has been pending or in flight for `idle` seconds"""
        inflight, last = set(), time.monotonic()
        try:
            while True:
                for tid, spec in self._claim():
                    self.claimed.append(tid)
                    try:
                        self.backend.submit(tid, spec)
                        inflight.add(tid)
                    except Exception:
                        self._finish(tid, 1)
                    last = time.monotonic()
                for tid, status in self.backend.poll():
                    if tid in inflight:
                        inflight.discard(tid)
                        self._finish(tid, status)
                        last = time.monotonic()
                if inflight:
                    last = time.monotonic()
                elif time.monotonic() - last >= self.idle:
                    return
                time.sleep(self.poll)
        finally:
            close = getattr(self.backend, "close", None)
            if close is not None:
                close()


def spool_run(spec, spool_dir, make_backend, idle=2.0, poll=0.02, timeout=None):
    """One invocation: spool `spec` (a JSON-able dict, e.g. {"argv0": ..., "argv": [...]}) and return its exit
    status, serving the spool (with make_backend()) whenever no other process does."""
    os.makedirs(spool_dir, exist_ok=True)
    tid = f"{os.getpid()}-{uuid.uuid4().hex[:10]}"
    task = os.path.join(spool_dir, tid + ".task")
    done = os.path.join(spool_dir, tid + ".done")
    _atomic_write(task, json.dumps(spec))
    t0 = time.monotonic()
    with open(os.path.join(spool_dir, "server.lock"), "a") as lockf:
        while True:
            if os.path.exists(done):
                with open(done) as f:
                    status = int(f.read().strip() or 1)
                os.remove(done)
                return status
            if timeout is not None and time.monotonic() - t0 > timeout:
                raise TimeoutError(f"spooled task {tid} not finished after {timeout} s")
            try:
                fcntl.flock(lockf, fcntl.LOCK_EX | fcntl.LOCK_NB)
            except OSError:
                time.sleep(poll)
                put_back_if_orphaned(spool_dir, tid)
                continue
            try:
                put_back_if_orphaned(spool_dir, tid)
                SpoolServer(spool_dir, make_backend(), idle=idle, poll=poll).serve()
            finally:
                fcntl.flock(lockf, fcntl.LOCK_UN)


def put_back_if_orphaned(spool_dir, tid):
    """if task tid is claimed by a process that is gone and has no status yet, make it pending again"""
    if os.path.exists(os.path.join(spool_dir, tid + ".task")) or os.path.exists(os.path.join(spool_dir, tid + ".done")):
        return False
    for f in os.listdir(spool_dir):
        if f.startswith(tid + ".claimed."):
            pid = int(f.rsplit(".", 1)[1])
            if not pid_alive(pid):
                try:
                    os.rename(os.path.join(spool_dir, f), os.path.join(spool_dir, tid + ".task"))
                    return True
                except OSError:
                    return False
    return False


class ServingBackend:
    """Backend of the GPU serving loop: prepare(spec) -> (group, dropin task, M) runs on a host thread pool (the
    CPU setup of one task overlaps the GPU work of others), the task goes to serve.Server (continuous batching
    by operator, admission by HBM footprint), and finish(spec, result) writes its output files and returns the
    exit status; any exception gives status 1 (the caller may then run the official binary for that task)."""

    def __init__(self, server, prepare, finish, threads=4):
        from concurrent.futures import ThreadPoolExecutor
        self.server, self.prepare, self.finish = server, prepare, finish
        self.pool = ThreadPoolExecutor(threads)
        self.lock = threading.Lock()
        self.done = []

    def submit(self, tid, spec):
        self.pool.submit(self._run, tid, spec)

    def _run(self, tid, spec):
        try:
            group, task, M = self.prepare(spec)
            req = self.server.submit(group, task, M)
            status = self.finish(spec, self.server.wait(req))
        except Exception:
            status = 1
        with self.lock:
            self.done.append((tid, status))

    def poll(self):
        with self.lock:
            out, self.done = self.done, []
        return out

    def close(self):
        self.pool.shutdown(wait=True)
