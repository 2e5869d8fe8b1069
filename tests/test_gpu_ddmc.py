"""DDMC-style leakage in optically thick cells (RadiationIMCParameters::withDDMC,
radiation/RadiationIMC.hpp:1282-1612) on the GPU against the reference.

* Recorded reference segments (tests/golden/replay_ddmc*.npz: a gray step
  cube with DDMC; the same with Random Walk taking the deeper particles; a
  64-group cube with DDMC in its multigroup PGRW form) replay with the same
  event, destination cell and draw count, the same DDMC/Random Walk choice,
  and positions, directions, weights and tallies to the replay tolerances.
  The fixtures hold DDMC census events and leaks through every kind of face.
* Whole steps conserve energy, agree with the reference's serial path within
  the seed-to-seed scatter, and the FP32-tracking form agrees with the FP64 form.
"""
import numpy as np
import pytest

from conftest import golden
from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine

from test_gpu_parity import _check_replay, close

pytestmark = pytest.mark.gpu


def _mg_ddmc(seed=13, precision=A.PRECISION_FP64, n=6):
    p = problems.mg_cube(n=n, groups=64, kappa0=1e-4, new_photons_per_cell=3, comb_nmin=3, seed=seed, dt=1e-10,
                         with_random_walk=False, precision=precision)
    p.sigma_s = np.full(p.ncells, 1000.0)
    p.with_ddmc = True
    p.ddmc_use_multigroup_pgrw = True
    return p


FIXTURES = {
    "replay_ddmc.npz": lambda: problems.ddmc_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20, seed=11),
    "replay_ddmc_rw.npz": lambda: problems.ddmc_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20,
                                                     seed=12, with_random_walk=True,
                                                     rw_min_particle_optical_depth=20.0),
    "replay_ddmc_mg.npz": _mg_ddmc,
}


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_ddmc_replay_matches_reference(oracle_lib, name):
    g = golden(name)
    p = FIXTURES[name]()
    e = Engine(p)
    e.set_cell_state(g["T_start"], None, None)
    e.phase("prestep", p.dt)
    freq = g["freq_before"] if "freq_before" in g else None
    b = oracle_lib.ReplayBatch(g["before"], g["cell"], g["tape_offset"], g["tape_length"], g["tape"],
                               frequency=freq)
    e.replay(b)
    _check_replay(b, g, p.ncells, time_rel=1e-13)
    np.testing.assert_array_equal(b["used_random_walk"], g["used_rw"])
    ddmc = g["used_rw"] == 2
    leaks = ddmc & (g["status"] == 1)
    assert ddmc.sum() > 500 and leaks.sum() > 100 and (ddmc & (g["status"] == 2)).sum() > 100
    # leaks through faces of every axis and both orientations
    sides = set()
    for q in np.where(leaks)[0]:
        d = int(g["next"][q]) - int(g["cell"][q])
        sides.add(d)
    assert len(sides) == 6, sides
    if freq is not None:
        ok = b["phys_status"] == g["status"]
        assert close(b["phys_frequency"][ok], g["freq_after"][ok], 1e-12).all()
    e.close()


def _balance(st):
    src = st["energy_census_in"] + st["energy_emitted"]
    sink = st["energy_deposited"] + st["energy_escaped"] + st["energy_census_pre_comb"]
    return abs(src - sink) / max(src, 1e-300)


@pytest.mark.parametrize("precision", [A.PRECISION_FP64, A.PRECISION_FP32_TRACK])
def test_ddmc_energy_conservation(precision):
    for p in (problems.ddmc_cube(n=12, precision=precision), _mg_ddmc(precision=precision, n=8)):
        e = Engine(p)
        for _ in range(3):
            st = e.step()
            assert _balance(st) < 1e-10
        e.close()


def test_ddmc_steps_statistics_vs_reference(ref_lib):
    """Four steps of a DDMC cube on independent seeds: the GPU and the
    reference's serial path agree cell by cell under the batch gate."""
    from batchcheck import assert_agree, run_batch

    def prob(s):
        return problems.ddmc_cube(n=8, new_photons_per_cell=4, face_packets=80, comb_nmin=20, seed=s)
    assert_agree(run_batch(Engine, prob, range(20, 36), 4), run_batch(ref_lib.Reference, prob, range(60, 76), 4),
                 "DDMC cube 8^3: engine vs reference")


def test_ddmc_fp32_tracking_agrees_with_fp64():
    from batchcheck import assert_agree, run_batch

    def prob(precision):
        return lambda s: problems.ddmc_cube(n=10, new_photons_per_cell=4, face_packets=80, comb_nmin=20, seed=s,
                                            precision=precision)
    assert_agree(run_batch(Engine, prob(A.PRECISION_FP32_TRACK), range(30, 46), 4),
                 run_batch(Engine, prob(A.PRECISION_FP64), range(70, 86), 4), "DDMC cube 10^3: FP32 vs FP64")
