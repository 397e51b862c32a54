"""Writes tests/golden/dropin_write.json by running the reference's own writer (BlocksviBe's cli._write ->
_write_one -> _rows -> b3djson.write_spin, read from REFERENCE) on results in the form the drop-in returns
(blocksvibe_b200.dropin.task_results with OutputInfo objects), for the cases of dropin_cases.py: every spin file
of two blocks_3d invocations per case, plus the task attributes the file header prints.  That the reference's
writer consumes these results at all is the point; the bytes pin the GPU writer (jsonout.SpinWriter).

    python tests/golden/make_dropin_golden.py REFERENCE
"""
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import ref_standins                                          # noqa: E402

HEADER_ATTRS = ("two_js", "two_j12", "two_j43", "delta_12", "delta_43", "delta_1_plus_2", "q4", "sign", "order",
                "Lambda", "kept_pole_order", "coordinates", "precision", "two_js_internal", "out_template", "argv")


def consumer_files(cli, case):
    """{q: {two_j: text}} of the reference writer on the drop-in's results, and the tasks' header attributes"""
    import dropin_cases as DC
    from blocksvibe_b200 import dropin as DI
    vals, outputs, Sm, L = DC.host_values(case)
    pp = case[4]
    with tempfile.TemporaryDirectory() as d:
        tasks = [cli.Task(DC.argv(case, q4, d)) for q4 in DC.Q4S]
        d12 = tasks[0].delta_1_plus_2
        infos = {(c, d12): DI.OutputInfo(outputs[c]) for c in vals}
        tjs = sorted(tasks[0].two_js_internal)
        per_task = DI.task_results(tjs, pp, {(c, d12): mv for c, mv in vals.items()}, infos, Sm, L, len(tasks))
        results = {(tuple(t.q4), t.sign): r for t, r in zip(tasks, per_task)}
        cli._write(tasks, results)
        files = {}
        for q, t in enumerate(tasks):
            files[q] = {}
            for tj in t.two_js_internal:
                with open(t.path(tj / 2.0)) as f:
                    files[q][tj] = f.read()
        attrs = [{a: sorted(getattr(t, a)) if a == "coordinates" else getattr(t, a) for a in HEADER_ATTRS}
                 for t in tasks]
        for a in attrs:
            a["out_template"] = a["out_template"].replace(d, "OUT")
            a["argv"] = [x.replace(d, "OUT") for x in a["argv"]]
        for q in files:
            for tj in files[q]:
                files[q][tj] = files[q][tj].replace(d, "OUT")
    return files, attrs


def main(reference):
    ref_standins.install(reference)
    from blocksvibe import cli
    import json_cases as JC
    out = []
    for ci, case in enumerate(JC.SPIN_CASES):
        files, attrs = consumer_files(cli, case)
        out.append({"case": ci, "tasks": attrs,
                    "files": {str(q): {str(tj): t for tj, t in f.items()} for q, f in files.items()}})
    path = os.path.join(HERE, "dropin_write.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
