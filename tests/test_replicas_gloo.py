"""The multi-GPU plumbing of bench.py (replicas only: no data-path collective) on CPU with two gloo ranks:
the process group comes up, the barrier passes, and every rank sees the maximum of the ranks' timings."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank), B3D_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup()
    bench.barrier(w)
    out[r] = bench.max_over_ranks(10.0 + r, w, "cpu")
    dist.destroy_process_group()


def test_two_gloo_ranks_max_timing():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 11.0, 1: 11.0}

