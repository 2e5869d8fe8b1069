"""Online tuning of the transport kernel's refill burst
(storm_cuda_autotune_transport): it runs its schedule of candidates, keeps one
of them, and changes no result."""
import numpy as np
import pytest

from storm_b200 import problems
from storm_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _run(problem, steps, tune):
    e = Engine(problem)
    seen = []
    if tune:
        e.autotune_transport(1)
    for _ in range(steps):
        seen.append(e.transport_burst())
        e.step()
    final = e.transport_burst()
    T = e.cells()["temperature"]
    e.close()
    return T, seen, final


def test_autotune_keeps_a_candidate_and_changes_no_result():
    p = problems.uniform_cube(n=12, kappa=50.0, packets_per_step=2e4, seed=31)
    T0, seen0, final0 = _run(p, 11, tune=False)
    T1, seen1, final1 = _run(p, 11, tune=True)
    assert all(not t for _, t in seen0) and final0[0] == 8   # gray Cartesian default
    # the schedule: 1 2 4 8 16 16 8 4 2 1, one step each, then the kept burst
    assert [b for b, _ in seen1[:10]] == [1, 2, 4, 8, 16, 16, 8, 4, 2, 1]
    assert all(t for _, t in seen1[:10]) and not seen1[10][1]
    assert final1[0] in (1, 2, 4, 8, 16) and not final1[1]
    # the burst only reorders the FP64 tally sums
    np.testing.assert_allclose(T1, T0, rtol=1e-7)


def test_autotune_can_be_stopped():
    p = problems.uniform_cube(n=8, kappa=5.0, packets_per_step=5e3, seed=32)
    e = Engine(p)
    e.autotune_transport(2)
    e.step()
    e.step()
    e.step()
    assert e.transport_burst() == (2, True)
    e.autotune_transport(0)
    assert e.transport_burst() == (2, False)
    e.step()
    e.close()
