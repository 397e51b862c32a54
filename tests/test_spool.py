"""The spool front end (blocksvibe_b200.spool) with concurrent client processes and a host-only fake backend
(CPU only): every invocation gets its exit status, one process serves at a time and admits tasks while others
run (no quiet window), a task whose serving process died is put back and run by the next one, and a failing
task fails alone."""
import json
import multiprocessing
import os
import sys
import time

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
import spool_fakes as SF  # noqa: E402


def _run(tmp_path, specs, delays, crash_after=None, idle=0.5):
    d, out = str(tmp_path / "spool"), str(tmp_path / "out")
    os.makedirs(out)
    log = str(tmp_path / "batches.jsonl")
    ctx = multiprocessing.get_context("spawn")
    procs = []
    for i, (spec, delay) in enumerate(zip(specs, delays)):
        ca = crash_after if i == 0 else None
        p = ctx.Process(target=SF.client, args=(d, spec, log, out, str(tmp_path / f"r{i}"), idle, ca, delay))
        p.start()
        procs.append(p)
    for p in procs:
        p.join(90)
        assert not p.is_alive()
    batches = [json.loads(x) for x in open(log)] if os.path.exists(log) else []
    status = {}
    for i in range(len(specs)):
        r = tmp_path / f"r{i}"
        status[i] = int(r.read_text()) if r.exists() else None
    return status, batches, out, procs


def test_concurrent_invocations_share_one_serving_loop(tmp_path):
    n = 6
    specs = [{"argv0": "blocks_3d", "argv": ["-p", f"task{i}"], "name": f"t{i}"} for i in range(n)]
    status, batches, out, _ = _run(tmp_path, specs, [0.15 * i for i in range(n)])
    assert status == {i: 0 for i in range(n)}
    ran = [t for b in batches for t in b["tasks"]]
    assert sorted(ran) == sorted(s["name"] for s in specs)          # every task exactly once
    for s in specs:
        assert len(open(os.path.join(out, s["name"] + ".out")).read().split()) == 1
    assert len(batches) >= 2                                        # later arrivals joined later batches
    last_submit = max(float((tmp_path / f"r{i}.submitted").read_text()) for i in range(n))
    assert batches[0]["start"] < last_submit                        # the first batch ran before the last arrival
    # one serving process at a time: batches of different processes never overlap in time
    for a in batches:
        for b in batches:
            if a["pid"] != b["pid"]:
                assert a["end"] <= b["start"] or b["end"] <= a["start"]


def test_dead_serving_process_tasks_are_put_back(tmp_path):
    """the first client serves and dies (os._exit) after claiming tasks of others; those tasks are put back by
    their clients and run by the next serving process"""
    n = 5
    specs = [{"argv0": "blocks_3d", "argv": [f"t{i}"], "name": f"t{i}"} for i in range(n)]
    status, batches, out, procs = _run(tmp_path, specs, [0.0] + [0.05] * (n - 1), crash_after=2)
    assert procs[0].exitcode == 17
    assert all(status[i] == 0 for i in range(1, n))
    ran = [t for b in batches for t in b["tasks"]]
    assert sorted(ran) == sorted(f"t{i}" for i in range(1, n))        # the dead process ran nothing
    assert all(b["pid"] != procs[0].pid for b in batches)


def test_failing_task_fails_alone(tmp_path):
    specs = [{"argv0": "blocks_3d", "argv": [f"t{i}"], "name": f"t{i}", "fail": i == 1} for i in range(3)]
    status, _, _, _ = _run(tmp_path, specs, [0.0, 0.02, 0.04])
    assert status == {0: 0, 1: 3, 2: 0}


def test_orphan_put_back_only_for_dead_owners(tmp_path):
    from blocksvibe_b200 import spool
    d = str(tmp_path)
    open(os.path.join(d, f"a.claimed.{os.getpid()}"), "w").close()         # claimed by a live process
    assert not spool.put_back_if_orphaned(d, "a")
    ctx = multiprocessing.get_context("spawn")
    p = ctx.Process(target=time.sleep, args=(0,))
    p.start()
    p.join()
    open(os.path.join(d, f"b.claimed.{p.pid}"), "w").close()              # claimed by a process that is gone
    assert spool.put_back_if_orphaned(d, "b")
    assert os.path.exists(os.path.join(d, "b.task"))
