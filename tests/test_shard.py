"""One IMC problem split over ranks by particle shards, on the CPU: the oracle
(the C restatement of the path) run as two `gloo` ranks holding one shard
each, against one instance holding both shards.  The exchange is the
callback storm_cuda_set_sharding documents (an in-place sum over the ranks,
here torch.distributed.all_reduce on gloo).

For a given number of shards the step's results do not depend on how the
shards are spread over ranks, up to the summation order of the tallies:
counts (emitted, census, segments, escapes) exact, the census particle for
particle, the cell state to 1e-12.  Also: one shard is the unsharded step,
and two shards agree with the unsharded run within statistics.
"""
import os
import socket

import numpy as np
import pytest

STEPS = 3
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "time_left", "weight", "initial_weight")


def _problem(kind, seed=7):
    from storm_b200 import problems
    if kind == "slab":
        return problems.gray_slab(nx=30, new_photons_per_cell=8, face_packets=1500, comb_nmin=40, seed=seed)
    return problems.step_cube(n=6, new_photons_per_cell=4, face_packets=40, comb_nmin=12, seed=seed)


def _run(problem, shards, lo, hi, exchange=None, steps=STEPS):
    from oracle import orc
    o = orc.Oracle(problem)
    o.set_sharding(shards, lo, hi, exchange)
    stats = [o.step() for _ in range(steps)]
    cells = o.cells()
    cen = o.census()
    out = {"stats": stats, "cells": {k: cells[k] for k in ("temperature", "internal_energy", "erad_time_avg",
                                                          "erad_census")},
           "census": {f: getattr(cen, f) for f in FIELDS + ("cell",)}}
    o.close()
    return out


def _rank_main(rank, world, port, kind, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def exchange(values):
            t = torch.from_numpy(values)   # shares the oracle's buffer
            dist.all_reduce(t)
        q.put((rank, _run(_problem(kind), world, rank, rank + 1, exchange)))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.fixture(scope="module")
def oracle_built(oracle_lib):
    return oracle_lib


@pytest.mark.parametrize("kind", ["slab", "cube"])
def test_two_ranks_give_the_two_shard_result(oracle_built, kind):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, kind, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, out = q.get(timeout=300)
        res[r] = out
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    one = _run(_problem(kind), 2, 0, 2)
    # counts: the two ranks' sums equal the one instance's, step by step
    for s in range(STEPS):
        for k in ("emitted_cells", "emitted_faces", "census_in", "census_out_pre_comb", "census_out", "segments",
                  "escaped", "cutoff", "rw_steps"):
            assert res[0]["stats"][s][k] + res[1]["stats"][s][k] == one["stats"][s][k], (s, k)
    # the cell state is the same on both ranks and on the one instance
    for k, v in one["cells"].items():
        for r in (0, 1):
            np.testing.assert_allclose(res[r]["cells"][k], v, rtol=1e-12, atol=0, err_msg=k)
    # the census: rank 0 holds shard 0's part, rank 1 shard 1's, in the one instance's order
    for f in FIELDS + ("cell",):
        joined = np.concatenate([res[0]["census"][f], res[1]["census"][f]])
        if f == "cell":
            np.testing.assert_array_equal(joined, one["census"][f])
        else:
            # the cell state differs in the last bits (tally summation order), and a
            # particle's later segments inherit that through the Fleck factor
            np.testing.assert_allclose(joined, one["census"][f], rtol=1e-9, atol=1e-12, err_msg=f)


def test_one_shard_is_the_unsharded_step(oracle_built):
    from oracle import orc
    p = _problem("cube")
    a = _run(p, 1, 0, 1)
    o = orc.Oracle(_problem("cube"))
    for _ in range(STEPS):
        o.step()
    c = o.cells()
    for k, v in a["cells"].items():
        np.testing.assert_array_equal(v, c[k], err_msg=k)
    o.close()


def test_sharded_runs_agree_with_unsharded_within_statistics(oracle_built):
    """Two shards change which particles the comb keeps (teeth restart at each
    shard's run), not the expectation: over independent seeds, per-cell
    quantities agree with the unsharded step under the batch gate."""
    from oracle import orc
    from storm_b200 import batchstats
    steps = 4

    def batch(shards, seeds):
        runs = []
        for s in seeds:
            p = _problem("cube", seed=s)
            o = orc.Oracle(p)
            o.set_sharding(shards, 0, shards)
            runs.append(batchstats.run_snapshots(o, p, steps, (steps,)))
            o.close()
        return np.array(runs)
    res = batchstats.compare(batch(2, range(100, 116)), batch(1, range(200, 216)))
    assert res["all"]["tests"] > 0 and res["passed"], res["all"] | {"totals": res["totals"]}
