"""The bench's multi-rank plumbing on CPU: two gloo ranks set up from the
torchrun environment, the max-over-ranks and sum reductions the timing and
the whole-job totals use, and the barrier.  (The GPU arm uses the same calls
over NCCL.)"""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import types
    import bench
    got_ws, got_rank, local, dist = bench.dist_setup(types.SimpleNamespace(impl="reference"))
    mx = bench.reduce(dist, 10.0 + rank, "max", "reference")
    total = bench.reduce(dist, 1.0 + rank, "sum", "reference")
    bench.barrier(dist, "reference")
    out.put((got_rank, got_ws, local, mx, total))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_meet():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    assert res == [(0, 2, 0, 11.0, 3.0), (1, 2, 1, 11.0, 3.0)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import types
    import bench
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        ws, rank, local, dist = bench.dist_setup(types.SimpleNamespace(impl="reference"))
        assert (ws, rank, local, dist) == (1, 0, 0, None)
        assert bench.reduce(dist, 4.5, "max", "reference") == 4.5
        bench.barrier(dist, "reference")
    finally:
        os.environ.update(env)
