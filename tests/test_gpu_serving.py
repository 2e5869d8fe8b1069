"""The serving loop (storm_server_*): independent problems admitted by slots
and an HBM budget and advanced concurrently give the same results as each
problem run alone, and every request completes."""
import numpy as np
import pytest

from storm_b200 import problems
from storm_b200.engine import Engine, Server

pytestmark = pytest.mark.gpu


def _alone(problem, steps):
    e = Engine(problem)
    segs = 0
    for _ in range(steps):
        segs += e.step()["segments"]
    T = e.cells()["temperature"]
    e.close()
    return T, segs


def test_results_same_alone_and_in_the_mix():
    mix = problems.serving_mix(10, n_range=(8, 24), packets_range=(2e3, 5e4), steps_range=(2, 6), seed=3)
    srv = Server(max_active=4, workers=4)
    tickets = {srv.submit(p, s): (p, s) for p, s in mix}
    srv.drain()
    res = srv.poll()
    st = srv.stats()
    srv.close()
    assert len(res) == len(mix) and st["completed"] == len(mix) and st["failed"] == 0
    for r in res:
        p, s = tickets[r["ticket"]]
        assert r["status"] == 0 and r["steps"] == s
        T, segs = _alone(p, s)
        # tallies are summed with atomics: the material state may differ in the
        # last bits between two runs, and with it rare event decisions
        np.testing.assert_allclose(r["temperature"], T, rtol=1e-9)
        assert abs(r["segments"] - segs) <= 1e-6 * segs + 2


def test_admission_respects_slots_and_budget():
    mix = problems.serving_mix(6, n_range=(8, 16), packets_range=(2e3, 1e4), steps_range=(2, 3), seed=5)
    srv = Server(max_active=2, workers=3, hbm_budget_bytes=1 << 30)
    for p, s in mix:
        srv.submit(p, s, want_temperature=False)
    srv.drain()
    st = srv.stats()
    res = srv.poll()
    srv.close()
    assert st["completed"] == 6 and len(res) == 6
    # admitted requests (their estimates while being created, then their
    # actual bytes) never exceeded the budget
    assert st["peak_device_bytes"] <= st["budget_bytes"] == 1 << 30
    # with two slots, later requests waited in the queue
    assert max(r["queued_ms"] for r in res) > 0.0


def test_reused_streams_and_memory_give_the_same_result():
    """A handle created on streams, events, page-locked buffers and device
    memory that earlier handles of other sizes used (and released) runs its
    problem exactly as the first handle did, and a repeated request of a size
    the cache holds makes no new device allocation."""
    from storm_b200.engine import pool_counters
    p = problems.uniform_cube(n=12, kappa=50.0, packets_per_step=2e4, seed=21)
    T0, segs0 = _alone(p, 3)
    for q, _ in problems.serving_mix(4, n_range=(8, 20), packets_range=(2e3, 3e4), steps_range=(1, 2), seed=9):
        _alone(q, 1)
    before = pool_counters()
    T1, segs1 = _alone(p, 3)
    after = pool_counters()
    np.testing.assert_allclose(T1, T0, rtol=1e-9)
    assert abs(segs1 - segs0) <= 1e-6 * segs0 + 2
    assert after["mallocs"] == before["mallocs"]
    assert after["live_bytes"] == before["live_bytes"]


def test_release_cached_returns_the_cache():
    """storm_cuda_release_cached hands the cached device blocks back to the
    driver; a later handle allocates afresh and still runs."""
    from storm_b200.engine import pool_counters, release_cached
    p = problems.uniform_cube(n=10, kappa=5.0, packets_per_step=1e4, seed=4)
    T0, _ = _alone(p, 2)
    released = release_cached(0)
    c = pool_counters()
    assert released > 0 and c["cached_bytes"] == 0 and c["live_bytes"] == 0
    T1, _ = _alone(p, 2)
    np.testing.assert_allclose(T1, T0, rtol=1e-9)
    assert pool_counters()["mallocs"] > c["mallocs"]
