"""Checkpoint and restore of a handle's step-to-step state (census bank, cell
state, face temperatures, step counter): a run interrupted after two steps and
resumed from its checkpoint in a fresh handle repeats the uninterrupted run.
Tallies are summed with atomics, so temperatures agree to 1e-9 rather than bit
for bit."""
import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, StormError

pytestmark = pytest.mark.gpu

CASES = {
    "cube_fp64": lambda: problems.step_cube(n=16, new_photons_per_cell=3, face_packets=60, comb_nmin=10),
    "cube_fp32": lambda: problems.step_cube(n=16, new_photons_per_cell=3, face_packets=60, comb_nmin=10,
                                            precision=A.PRECISION_FP32_TRACK),
    "mg_fp32": lambda: problems.mg_cube(n=6, groups=64, kappa0=1.0, new_photons_per_cell=4, comb_nmin=4,
                                        precision=A.PRECISION_FP32_TRACK),
    "voronoi_fp64": lambda: problems.voronoi_cube(ncells=300, packets_per_step=2e4, seed=3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_resume_from_checkpoint_repeats_the_run(name):
    p = CASES[name]()
    a = Engine(p)
    for _ in range(4):
        a.step()
    Ta, na = a.cells()["temperature"], a.census_count()
    a.close()
    b = Engine(p)
    for _ in range(2):
        b.step()
    blob = b.checkpoint()
    b.close()
    c = Engine(p)
    c.restore(blob)
    for _ in range(2):
        c.step()
    Tc, nc = c.cells()["temperature"], c.census_count()
    assert abs(int(nc) - int(na)) <= 1e-3 * na
    np.testing.assert_allclose(Tc, Ta, rtol=1e-9)
    c.close()


def test_checkpoint_rejects_another_problem():
    a = Engine(problems.step_cube(n=8))
    a.step()
    blob = a.checkpoint()
    a.close()
    other = Engine(problems.step_cube(n=10))
    with pytest.raises(StormError):
        other.restore(blob)
    with pytest.raises(StormError):
        other.restore(blob[:40])
    other.close()
