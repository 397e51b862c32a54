"""A host-only stand-in for the GPU backend of the spool front end (blocksvibe_b200.spool), for the CPU tests:
it runs the claimed tasks in batches on a worker thread (a batch = every task submitted while the previous
batch ran: continuous batching), records each batch as a JSON line, and writes one output file per task."""
import json
import os
import threading
import time

from blocksvibe_b200 import spool


class FakeBackend:
    def __init__(self, log_path, out_dir, run_s=0.3, crash_after=None):
        self.log_path, self.out_dir, self.run_s, self.crash_after = log_path, out_dir, run_s, crash_after
        self.lock = threading.Condition()
        self.waiting, self.done, self.nsub, self.stop = [], [], 0, False
        self.th = threading.Thread(target=self._loop, daemon=True)
        self.th.start()

    def submit(self, tid, spec):
        with self.lock:
            self.nsub += 1
            if self.crash_after is not None and self.nsub > self.crash_after:
                os._exit(17)                                  # the serving process dies with tasks claimed
            self.waiting.append((tid, spec, time.time()))
            self.lock.notify_all()

    def _loop(self):
        while True:
            with self.lock:
                while not self.waiting and not self.stop:
                    self.lock.wait(0.01)
                if self.stop and not self.waiting:
                    return
                batch, self.waiting = self.waiting, []
            t0 = time.time()
            time.sleep(self.run_s)                            # the "GPU run" of the batch
            with open(self.log_path, "a") as f:
                f.write(json.dumps({"pid": os.getpid(), "start": t0, "end": time.time(),
                                    "tasks": [s["name"] for _, s, _ in batch]}) + "\n")
            res = []
            for tid, spec, _ in batch:
                with open(os.path.join(self.out_dir, spec["name"] + ".out"), "a") as f:
                    f.write(f"{os.getpid()}\n")
                res.append((tid, 3 if spec.get("fail") else 0))
            with self.lock:
                self.done += res

    def poll(self):
        with self.lock:
            out, self.done = self.done, []
        return out

    def close(self):
        with self.lock:
            self.stop = True
            self.lock.notify_all()
        self.th.join()


def client(spool_dir, spec, log_path, out_dir, result_path, idle=0.5, crash_after=None, delay=0.0):
    time.sleep(delay)
    with open(result_path + ".submitted", "w") as f:
        f.write(str(time.time()))
    status = spool.spool_run(spec, spool_dir, lambda: FakeBackend(log_path, out_dir, crash_after=crash_after),
                             idle=idle, poll=0.01, timeout=60)
    with open(result_path, "w") as f:
        f.write(str(status))
