"""The serving loop: requests of two operators submitted together, admitted under an HBM budget that holds only
part of them, batched per operator and run by two workers on their own streams; every result is bit for bit the
result of the same task run alone, the admitted footprint never exceeds the budget, and batches mix requests."""
import numpy as np
import pytest

from test_gpu_dropin import make_group
from blocksvibe_b200 import dropin as DI, serve

pytestmark = pytest.mark.gpu


def test_serving_same_alone_and_in_the_mix(cuda):
    G, tasks_a, M, _, _ = make_group(nq=3, seed=21, coords=("xt",), d12="2.3")
    _, tasks_b, _, _, _ = make_group(nq=2, seed=22, coords=("xt",), d12="0")
    items = [(G, t, M) for t in tasks_a + tasks_b]
    # budget: room for about two requests at a time
    probe = DI.Operator(G, tasks_a[0].pp, tasks_a[0].parity, M, tasks_a[0].two_js_internal, ["xt"], ["2.3"], cuda)
    one = int(1.5 * probe.footprint_bytes(len(tasks_a[0].lambda_orders(G.Lambda))))
    srv = serve.Server(cuda, budget_bytes=2 * one + 1, workers=2, max_batch=8)
    try:
        reqs = [srv.submit(g, t, m) for g, t, m in items]
        for r in reqs:
            srv.wait(r, timeout=600)
    finally:
        srv.close()
    assert srv.peak_in_flight <= srv.budget
    assert any(len(ids) > 1 for _, ids in srv.batches)
    for r in reqs:
        alone = DI.run_group(G, [r.task], M, device=cuda, schedule="batched")
        k = (tuple(r.task.q4), r.task.sign)
        for c, (m, e) in alone[k][2].items():
            gm, ge = r.result[c]
            assert np.array_equal(m, gm) and np.array_equal(e, ge), (r.id, c)
    lat = srv.latencies()
    assert len(lat) == len(items) and all(x >= 0 for x in lat)


def test_poisson_replay_reports_latency(cuda):
    G, tasks, M, _, _ = make_group(nq=4, seed=23, coords=("xt_radial",), d12="6")
    srv = serve.Server(cuda, workers=2)
    try:
        reqs, elapsed = serve.replay(srv, [(G, t, M) for t in tasks], rate=50.0, seed=1)
    finally:
        srv.close()
    lat = [r.done - r.arrival for r in reqs]
    assert serve.percentile(lat, 0.5) <= serve.percentile(lat, 0.99)
    assert elapsed > 0 and all(r.result for r in reqs)


def test_device_resident_results_equal_host_results(cuda):
    """host_results=False leaves each result on the GPU (for the GPU JSON writer): same values"""
    G, tasks, M, _, _ = make_group(nq=3, seed=24, coords=("xt",), d12="2.3")
    out = {}
    for host in (True, False):
        srv = serve.Server(cuda, workers=2, max_batch=8, host_results=host)
        try:
            reqs = [srv.submit(G, t, M) for t in tasks]
            for r in reqs:
                srv.wait(r, timeout=600)
        finally:
            srv.close()
        out[host] = [r.result for r in reqs]
    for a, b in zip(out[True], out[False]):
        for key, (m, e) in a.items():
            x = b[key]
            assert np.array_equal(m, x.m.cpu().numpy()[:, :, :, :, 0]) and np.array_equal(e, x.e.cpu().numpy()[:, :, :, 0])
