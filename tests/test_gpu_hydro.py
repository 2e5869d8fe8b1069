"""Moving material (RadiationIMCParameters::withHydro) on the GPU against the
reference, whose cells carry a velocity and whose extensives carry a momentum.

* The prestep's Fleck factor with the cells' Lorentz factor
  (radiation/RadiationIMC.hpp:1636-1649) equals the reference's table.
* Recorded reference segments (tests/golden/replay_hydro*.npz: a gray cube
  with Random Walk and elastic scattering, a 64-group cube with PGRW, cells
  moving at up to 5 % of c) replay with the same event, destination cell and
  draw count, the same lab-frame direction, weight and frequency after
  Doppler-shifted opacities, comoving scatters and Random Walk jumps
  transformed back to the lab frame (:228-314, 1098-1110, 1252-1268,
  1700-1881), the same material and radiation tallies and the same momentum
  deposit per segment.
* With the cells at rest the moving-material kernels are the static ones: a
  whole step equals the oracle's on identical Philox streams.
* Whole steps with moving cells agree with the reference's serial path under
  the batch gate, momentum per cell included.
"""
import numpy as np
import pytest

from conftest import golden
from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, StormError

from test_gpu_parity import _check_replay, close

pytestmark = pytest.mark.gpu


def _problems():
    import sys
    from conftest import GOLDEN
    sys.path.insert(0, GOLDEN)
    import make_golden as MG
    return MG.hydro_problems(), MG.hydro_velocity


def _engine_at(p, g):
    e = Engine(p)
    e.set_cell_state(g["T_start"], None, None)
    e.set_cell_motion(velocity=g["vel_start"])
    e.phase("prestep", p.dt)
    return e


@pytest.mark.parametrize("name", ["replay_hydro.npz", "replay_hydro_mg.npz"])
def test_hydro_replay_matches_reference(oracle_lib, name):
    probs, _ = _problems()
    p = probs[name]
    g = golden(name)
    e = _engine_at(p, g)
    c = e.cells()
    assert close(c["fleck"], g["fleck"], 1e-12).all()
    assert close(c["sigma_a"], g["sigma_a"], 1e-12).all()
    mg = p.groups >= 2
    b = oracle_lib.ReplayBatch(g["before"], g["cell"], g["tape_offset"], g["tape_length"], g["tape"],
                               frequency=g["freq_before"] if mg else None, momentum=True)
    e.replay(b)
    _check_replay(b, g, p.ncells, time_rel=1e-13)
    ok = b["phys_status"] == g["status"]
    if mg:
        fa = g["freq_after"]
        assert close(b["phys_frequency"][ok], fa[ok], 1e-12).all()
    m = b["phys_momentum"].reshape(-1, 3)
    # the reference's deposits are differences of the cell's momentum before and
    # after the segment, so they carry that momentum's rounding: a few ulps of
    # mass |v| of the cell
    pcell = (p.mass[g["cell"]] * np.abs(g["vel_start"][g["cell"]]).max(1))[:, None]
    good = np.abs(m - g["momentum"]) <= 1e-12 * np.abs(g["momentum"]) + 4 * 2.2e-16 * pcell
    assert good[ok].all(), np.where(~good[ok].all(1))[0][:5]
    assert np.abs(g["momentum"]).max() > 0
    e.close()


def test_cells_at_rest_step_like_the_static_engine(oracle_lib):
    """A first step with every cell at rest is the static step (the Doppler
    factor is 1 and no frame transform applies); radiation then leaves momentum
    in the cells, which start to move."""
    p = problems.step_cube(n=10, new_photons_per_cell=3, face_packets=60, comb_nmin=10)
    p.with_hydro = True
    p.cell_velocity = np.zeros((p.ncells, 3))
    e, o = Engine(p), oracle_lib.Oracle(p)
    se, so = e.step(), o.step()
    for k in ("emitted_cells", "emitted_faces", "census_out", "segments", "escaped", "cutoff", "rw_steps"):
        assert se[k] == so[k], k
    ce, co = e.cells(), o.cells()
    assert close(ce["temperature"], co["temperature"], 1e-9).all()
    v, m = e.cell_motion()
    assert np.abs(m).max() > 0 and np.allclose(v, m / p.mass[:, None], rtol=1e-14, atol=0)
    assert (v[:, 0] > 0).mean() > 0.5   # pushed away from the hot x-low face
    e.close()


def test_moving_cells_agree_with_reference(ref_lib):
    """Four steps of the gray moving-material cube on independent seeds: per
    cell temperature, deposit, radiation energies and the momentum gained,
    engine against the reference's serial path under the batch gate."""
    from storm_b200 import batchstats
    from storm_b200.units import UNITS
    probs, vel = _problems()
    base = probs["replay_hydro.npz"]

    def prob(s):
        q = problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20, seed=s)
        q.sigma_s = base.sigma_s.copy()
        q.with_hydro = True
        q.cell_velocity = vel(q)
        return q

    def run(make, seeds):
        runs = []
        for s in seeds:
            q = prob(s)
            m = make(q)
            m0 = q.cell_velocity * q.mass[:, None]
            prev = m.cells()
            for _ in range(4):
                m.step()
                cur = m.cells()
                last = batchstats.step_quantities(prev, cur, q.volumes(), UNITS["arad"], UNITS["clight"], q.dt)
                prev = cur
            mom = (m.cell_motion() if isinstance(m, Engine) else m.motion())[1] - m0
            runs.append(np.concatenate([last, mom.T])[None])
            m.close()
        return np.array(runs)
    a = run(Engine, range(40, 56))
    b = run(ref_lib.Reference, range(80, 96))
    res = batchstats.compare(a[:, :, :4], b[:, :, :4])
    assert res["all"]["tests"] > 0 and res["passed"], res["all"] | {"totals": res["totals"]}
    sa, sb = batchstats.summarize(a[:, 0, 4:]), batchstats.summarize(b[:, 0, 4:])
    scale = np.maximum(np.abs(sa["mean"]), np.abs(sb["mean"])).max(axis=-1, keepdims=True)
    z, ok = batchstats.welch_z(sa, sb, batchstats.RESOLUTION * scale)
    gm = batchstats.gate(z[ok])
    assert gm["tests"] > 100 and gm["passed"], gm


def test_fp32_form_refuses_moving_material():
    p = problems.step_cube(n=4, precision=A.PRECISION_FP32_TRACK)
    p.with_hydro = True
    with pytest.raises(StormError):
        Engine(p)
