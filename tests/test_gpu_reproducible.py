"""Reproducible tallies (StormProblemDesc.reproducible_tallies): the transport's
material deposits and time-integrated radiation energy are summed per cell in
fixed point with integer atomics, so that a run repeats bit for bit.

* Two runs of one problem and seed give identical cell state and census,
  bit for bit, in both forms, gray and multigroup, on a Cartesian grid with
  Random Walk and DDMC and on a Voronoi mesh.
* The reproducible run is the same physics: against the oracle on identical
  Philox streams, counts exact and tallies to the usual 1e-9.
* Options whose tallies have no fixed-point sum are refused.
"""
import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, StormError
from storm_b200.mesh import build_voronoi

pytestmark = pytest.mark.gpu

CELLS = ("temperature", "internal_energy", "erad_time_avg", "erad_census")
COUNTS = ("emitted_cells", "emitted_faces", "census_out", "segments", "escaped", "cutoff", "rw_steps")


def _cube(precision):
    p = problems.step_cube(n=12, new_photons_per_cell=3, face_packets=60, comb_nmin=10, precision=precision)
    p.reproducible_tallies = True
    return p


def _mg(precision):
    p = problems.mg_cube(n=6, groups=64, kappa0=1.0, new_photons_per_cell=6, comb_nmin=6, seed=3, precision=precision)
    p.reproducible_tallies = True
    return p


def _ddmc(precision):
    p = problems.ddmc_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20, seed=11, precision=precision,
                           with_random_walk=True, rw_min_particle_optical_depth=20.0)
    p.reproducible_tallies = True
    return p


def _voronoi(precision):
    mesh = build_voronoi(np.random.default_rng(4).random((300, 3)) * 0.98 + 0.01)
    p = problems.voronoi_cube(ncells=300, packets_per_step=2e4, seed=4, mesh=mesh, precision=precision)
    p.reproducible_tallies = True
    return p


def _run(p, steps=3):
    e = Engine(p)
    stats = [e.step() for _ in range(steps)]
    cells = e.cells()
    census = e.census()
    e.close()
    return stats, cells, census


@pytest.mark.parametrize("precision", [A.PRECISION_FP64, A.PRECISION_FP32_TRACK])
@pytest.mark.parametrize("make", [_cube, _mg, _ddmc, _voronoi])
def test_runs_repeat_bit_for_bit(make, precision):
    s1, c1, p1 = _run(make(precision))
    s2, c2, p2 = _run(make(precision))
    for a, b in zip(s1, s2):
        for k in COUNTS:
            assert a[k] == b[k], k
        assert a["energy_deposited"] > 0
    for k in CELLS:
        np.testing.assert_array_equal(c1[k], c2[k], err_msg=k)
    assert p1.n == p2.n and p1.n > 0
    for f in ("x", "y", "z", "vx", "vy", "vz", "weight", "cell"):
        np.testing.assert_array_equal(getattr(p1, f), getattr(p2, f), err_msg=f)


def test_reproducible_step_matches_oracle(oracle_lib):
    p = _cube(A.PRECISION_FP64)
    e, o = Engine(p), oracle_lib.Oracle(p)
    for s in range(3):
        se, so = e.step(), o.step()
        for k in COUNTS:
            assert se[k] == so[k], (s, k)
        ce, co = e.cells(), o.cells()
        for k in CELLS:
            a, b = np.asarray(ce[k]), np.asarray(co[k])
            assert (np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), np.abs(b)) + 1e-300).all(), (s, k)
    e.close()
    o.close()


def test_unsupported_combinations_are_refused():
    hydro = _cube(A.PRECISION_FP64)
    hydro.with_hydro = True
    hydro.cell_velocity = np.zeros((hydro.ncells, 3))
    eg = _mg(A.PRECISION_FP64)
    eg.with_eg_time_avg = True
    nocomb = _cube(A.PRECISION_FP64)
    nocomb.comb_enabled = False
    for p in (hydro, eg, nocomb):
        with pytest.raises(StormError):
            Engine(p)
    e = Engine(_cube(A.PRECISION_FP64))
    with pytest.raises(StormError):
        e.set_sharding(2, 0, 1)
    e.close()
