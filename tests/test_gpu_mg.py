"""Multigroup (RadiationIMC<..., 64> with withMultigroupOpacity and PGRW) on the
GPU against the reference.

* The per-cell tables (Planck-mean opacity, Fleck factor) built from the same
  temperatures agree with the reference's to 1e-12.
* Recorded reference segments (tests/golden/replay_mg*.npz, with their
  frequencies and uniforms) replay with the same event, destination cell and
  draw count, the same frequency after the segment (effective scatters and
  PGRW upscatters re-sample it from the cell's spectrum) and positions,
  weights and tallies to the replay tolerances of the gray path.
* Whole steps agree with the reference's own serial path statistically and
  conserve energy.
"""
import numpy as np
import pytest

from conftest import golden
from storm_b200 import problems
from storm_b200.engine import Engine

from test_gpu_parity import _check_replay, close

pytestmark = pytest.mark.gpu

FIXTURES = {
    "replay_mg.npz": dict(n=6, groups=64, new_photons_per_cell=3, comb_nmin=3, seed=5),
    "replay_mg_thin.npz": dict(n=6, groups=64, kappa0=1.0, new_photons_per_cell=3, comb_nmin=3, seed=6,
                               group_constant=False),
}


def _engine_at(g, kw):
    p = problems.mg_cube(**kw)
    e = Engine(p)
    e.set_cell_state(g["T_start"], None, None)
    e.phase("prestep", p.dt)
    return p, e


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_mg_tables_match_reference(name):
    g = golden(name)
    p, e = _engine_at(g, FIXTURES[name])
    c = e.cells()
    assert close(c["sigma_a"], g["sigma_a"], 1e-12).all()
    assert close(c["fleck"], g["fleck"], 1e-12).all()
    e.close()


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_mg_replay_matches_reference(oracle_lib, name):
    g = golden(name)
    p, e = _engine_at(g, FIXTURES[name])
    b = oracle_lib.ReplayBatch(g["before"], g["cell"], g["tape_offset"], g["tape_length"], g["tape"],
                               frequency=g["freq_before"])
    e.replay(b)
    # the tables are rebuilt here from the same temperatures with CUDA's exp and
    # pow, so event times carry an ulp of difference; where timeLeft - dt
    # cancels, that ulp is relative to the starting timeLeft
    _check_replay(b, g, p.ncells, time_rel=1e-13)
    ok = b["phys_status"] == g["status"]
    good = close(b["phys_frequency"][ok], g["freq_after"][ok], 1e-12)
    assert good.all(), np.where(~good)[0][:5]
    changed = g["freq_after"] != g["freq_before"]
    assert changed.sum() > 100   # the fixture exercises frequency re-sampling
    e.close()


def _balance(st):
    src = st["energy_census_in"] + st["energy_emitted"]
    sink = st["energy_deposited"] + st["energy_escaped"] + st["energy_census_pre_comb"]
    return abs(src - sink) / max(src, 1e-300)


def test_mg_energy_conservation():
    e = Engine(problems.mg_cube(n=12, groups=64, kappa0=1.0, new_photons_per_cell=4, comb_nmin=4))
    for _ in range(3):
        st = e.step()
        assert _balance(st) < 1e-10
        assert st["rw_steps"] > 0
    c = e.census()
    g = problems.mg_cube(n=12).group_bounds
    assert (c.frequency >= g[0]).all() and (c.frequency <= g[-1]).all()
    e.close()


def test_mg_steps_statistics_vs_reference(ref_lib):
    """Four steps of a small multigroup cube on independent seeds: the GPU and
    the reference's serial path agree cell by cell under the batch gate."""
    from batchcheck import assert_agree, run_batch

    def prob(s):
        return problems.mg_cube(n=6, groups=64, kappa0=1.0, new_photons_per_cell=6, comb_nmin=6, seed=s)
    assert_agree(run_batch(Engine, prob, range(20, 36), 4), run_batch(ref_lib.Reference, prob, range(60, 76), 4),
                 "multigroup cube 6^3 x 64: engine vs reference")


def test_mg_fp32_tracking_conserves_and_agrees_with_fp64():
    """The FP32-tracking form of a multigroup problem: energy conserved per step
    and temperatures within the seed-to-seed scatter of the FP64 form."""
    from storm_b200 import _abi as A

    from batchcheck import assert_agree, run_batch

    def prob(precision):
        return lambda s: problems.mg_cube(n=8, groups=64, kappa0=1.0, new_photons_per_cell=6, comb_nmin=6, seed=s,
                                          precision=precision)

    def check(e, st):
        assert _balance(st) < 1e-10
        c = e.census()
        g = e.problem.group_bounds
        assert (c.frequency >= g[0] * (1 - 1e-6)).all() and (c.frequency <= g[-1] * (1 + 1e-6)).all()
    a = run_batch(Engine, prob(A.PRECISION_FP32_TRACK), range(30, 46), 4, check)
    b = run_batch(Engine, prob(A.PRECISION_FP64), range(70, 86), 4, check)
    assert_agree(a, b, "multigroup cube 8^3 x 64: FP32 vs FP64")
