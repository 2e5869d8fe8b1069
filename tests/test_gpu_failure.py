"""Failure detection on the device, made on the host side of the boundary: no
test here faults, traps or hangs the GPU.

* The history cap: a handle created with max_rounds x segments_per_visit of 2
  segments per history.  The transport kernel stops every longer history and
  raises STORM_DERR_HISTORY_CAP with the cell and particle; the step returns
  STORM_ERR_DEVICE with that word, and a fresh handle on the same device then
  steps normally.
* Census weights the comb must refuse (population/CombPopulationControl.hpp:
  108-142): a NaN, +inf or negative census weight survives transport (the
  weight cutoff compares |w| with the initial |w|,
  radiation/RadiationIMC.hpp:1497, 1812), reaches the comb and fails the step
  with STORM_DERR_COMB_WEIGHT, as the reference's serial manager throws
  "particle weight is not finite" / "is negative" on the same census.
"""
import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, Particles, StormError

pytestmark = pytest.mark.gpu

STORM_ERR_DEVICE = 4
DERR_HISTORY_CAP = 8
DERR_COMB_WEIGHT = 6


@pytest.mark.parametrize("precision", [A.PRECISION_FP64, A.PRECISION_FP32_TRACK])
def test_history_cap_fails_the_step_and_the_device_stays_usable(precision):
    p = problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=10, precision=precision)
    p.max_rounds, p.segments_per_visit = 1, 2
    e = Engine(p)
    with pytest.raises(StormError) as ei:
        for _ in range(3):
            e.step()
    err = ei.value
    assert err.status == STORM_ERR_DEVICE and err.derr == DERR_HISTORY_CAP, err
    assert err.cell < p.ncells
    e.close()
    ok = Engine(problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=10, precision=precision))
    for _ in range(2):
        st = ok.step()
    assert st["segments"] > 0 and st["census_out"] > 0
    assert np.isfinite(ok.cells()["temperature"]).all()
    ok.close()


def _census(p, weight):
    """Ten census particles at cell centres, travelling +y, one of them (in an
    optically thin cell, where it reaches census) with `weight`."""
    xc, yc, zc = p.cell_centers()
    n = 10
    q = Particles(n)
    cells = np.arange(n) * 7 % p.ncells
    q.x, q.y, q.z = xc[cells].copy(), yc[cells].copy(), zc[cells].copy()
    q.vy[:] = 2.99792458e10
    q.time_left[:] = p.dt
    q.weight[:] = 1e3
    q.weight[1] = weight
    q.initial_weight = np.abs(q.weight)
    q.cell = cells.astype(np.uint32)
    return q


@pytest.mark.parametrize("weight,message", [(np.nan, "not finite"), (np.inf, "not finite"), (-5.0, "negative")])
def test_bad_census_weight_fails_in_the_comb_like_the_reference(ref_lib, weight, message):
    p = problems.step_cube(n=6, new_photons_per_cell=2, face_packets=10, comb_nmin=4)
    e = Engine(p)
    e.set_census(_census(p, weight))
    with pytest.raises(StormError) as ei:
        e.step()
    assert ei.value.status == STORM_ERR_DEVICE and ei.value.derr == DERR_COMB_WEIGHT, ei.value
    e.close()
    r = ref_lib.Reference(p)
    r.set_census(_census(p, weight))
    with pytest.raises(RuntimeError, match=message):
        r.step()
    r.close()
