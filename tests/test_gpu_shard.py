"""One IMC problem split into particle shards on the GPU
(storm_cuda_set_sharding).

* The engine's sharded step against the oracle's (tests/test_shard.py pins
  the oracle's ranks against its single instance on the CPU): on identical
  Philox streams, counts exact and tallies to rounding, as for the unsharded
  step.
* Two handles holding one shard each, run side by side in two host threads on
  this GPU, against one handle holding both shards.  Their exchange is a host
  sum: each thread copies its buffer out, the two meet at a barrier, both add
  the same two buffers in the same order and copy the sum back.  No kernel
  waits on another handle's kernels; the threads wait on the host only.
  Counts exact, cell state and census to rounding.
"""
import threading

import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, device_array

pytestmark = pytest.mark.gpu

COUNTS = ("emitted_cells", "emitted_faces", "census_out_pre_comb", "census_out", "segments", "escaped", "cutoff",
          "rw_steps")
CELLS = ("temperature", "internal_energy", "erad_time_avg", "erad_census")


def _close(a, b, rel, atol=1e-300):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + atol


def _problem(kind, precision=A.PRECISION_FP64):
    if kind == "slab":
        return problems.gray_slab(new_photons_per_cell=5, face_packets=3000, comb_nmin=50, precision=precision)
    return problems.step_cube(n=12, new_photons_per_cell=3, face_packets=60, comb_nmin=10, precision=precision)


@pytest.mark.parametrize("kind", ["slab", "cube"])
def test_sharded_step_matches_oracle(oracle_lib, kind):
    p = _problem(kind)
    e = Engine(p)
    e.set_sharding(3, 0, 3)
    o = oracle_lib.Oracle(p)
    o.set_sharding(3, 0, 3)
    for s in range(3):
        se, so = e.step(), o.step()
        for k in COUNTS:
            assert se[k] == so[k], (s, k, se[k], so[k])
        ce, co = e.cells(), o.cells()
        for k in CELLS:
            assert _close(ce[k], co[k], 1e-9).all(), (s, k)
        pe, po = e.census(), o.census()
        assert pe.n == po.n
        np.testing.assert_array_equal(pe.cell, po.cell)
        for f in ("x", "y", "z", "weight") if pe.n else ():
            ok = _close(getattr(pe, f), getattr(po, f), 1e-12, atol=1e-14)
            assert ok.mean() > 0.999, (s, f, (~ok).sum())
    e.close()
    o.close()


class HostExchange:
    """The exchange of two handles on one GPU, summed on the host."""

    def __init__(self, ranks):
        self.barrier = threading.Barrier(ranks, timeout=120)
        self.slots = [None] * ranks

    def fn(self, rank):
        import torch

        def exchange(ptr, count, stream):
            buf = device_array(ptr, count)
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                self.slots[rank] = buf.cpu()          # waits for the handle's stream
                self.barrier.wait()
                total = self.slots[0].clone()
                for other in self.slots[1:]:
                    total += other
                self.barrier.wait()
                buf.copy_(total.to(buf.device))
                torch.cuda.current_stream().synchronize()
        return exchange


@pytest.mark.parametrize("precision", [A.PRECISION_FP64, A.PRECISION_FP32_TRACK])
@pytest.mark.parametrize("kind", ["slab", "cube"])
def test_two_handles_give_the_two_shard_result(kind, precision):
    steps = 3
    one = Engine(_problem(kind, precision))
    one.set_sharding(2, 0, 2)
    one_stats = [one.step() for _ in range(steps)]
    ex = HostExchange(2)
    engines = [Engine(_problem(kind, precision)) for _ in range(2)]
    for r, e in enumerate(engines):
        e.set_sharding(2, r, r + 1, ex.fn(r))
    stats = [[], []]
    errors = []

    def run(r):
        try:
            for _ in range(steps):
                stats[r].append(engines[r].step())
        except Exception as exc:   # reported below; the other thread's barrier times out
            errors.append(exc)
            ex.barrier.abort()
    threads = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for s in range(steps):
        for k in COUNTS:
            assert stats[0][s][k] + stats[1][s][k] == one_stats[s][k], (s, k)
    c1 = one.cells()
    for e in engines:
        c = e.cells()
        for k in CELLS:
            assert _close(c[k], c1[k], 1e-9).all(), k
    p1 = one.census()
    parts = [e.census() for e in engines]
    assert parts[0].n + parts[1].n == p1.n
    np.testing.assert_array_equal(np.concatenate([q.cell for q in parts]), p1.cell)
    for f in ("x", "y", "z", "weight") if p1.n else ():
        joined = np.concatenate([getattr(q, f) for q in parts])
        ok = _close(joined, getattr(p1, f), 1e-9, atol=1e-12)
        assert ok.mean() > 0.999, (f, (~ok).sum())
    for e in engines + [one]:
        e.close()
