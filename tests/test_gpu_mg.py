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
    the reference's serial path agree within the seed-to-seed scatter."""
    def run(make, seeds):
        out = []
        for s in seeds:
            p = problems.mg_cube(n=6, groups=64, kappa0=1.0, new_photons_per_cell=6, comb_nmin=6, seed=s)
            m = make(p)
            for _ in range(4):
                m.step()
            out.append(m.cells()["temperature"])
            m.close()
        return np.array(out)
    a = run(Engine, range(20, 28))
    b = run(ref_lib.Reference, range(60, 68))
    ma, mb = a.mean(0), b.mean(0)
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    z = np.abs(ma - mb) / np.maximum(se, 1e-9 * ma)
    assert (z < 4).mean() > 0.95, np.sort(z)[-10:]


def test_mg_fp32_tracking_conserves_and_agrees_with_fp64():
    """The FP32-tracking form of a multigroup problem: energy conserved per step
    and temperatures within the seed-to-seed scatter of the FP64 form."""
    from storm_b200 import _abi as A

    def run(precision, seeds):
        out = []
        for s in seeds:
            p = problems.mg_cube(n=8, groups=64, kappa0=1.0, new_photons_per_cell=6, comb_nmin=6, seed=s,
                                 precision=precision)
            e = Engine(p)
            for _ in range(4):
                st = e.step()
                assert _balance(st) < 1e-10
            c = e.census()
            assert (c.frequency >= p.group_bounds[0] * (1 - 1e-6)).all()
            assert (c.frequency <= p.group_bounds[-1] * (1 + 1e-6)).all()
            out.append(e.cells()["temperature"])
            e.close()
        return np.array(out)
    a = run(A.PRECISION_FP32_TRACK, range(30, 38))
    b = run(A.PRECISION_FP64, range(70, 78))
    ma, mb = a.mean(0), b.mean(0)
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    z = np.abs(ma - mb) / np.maximum(se, 1e-9 * ma)
    assert (z < 4).mean() > 0.95, np.sort(z)[-10:]
