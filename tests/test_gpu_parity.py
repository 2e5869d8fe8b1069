"""Parity of the CUDA engine (through the C ABI) with the reference and the oracle.

Tolerances:
  * integer / index work (event type, destination cell, draw counts, photon
    counts, census counts, comb counts): exact.
  * floating point of a single segment: 1e-12 relative (CUDA's log1p, expm1,
    sin, cos, exp, log may differ from glibc by an ulp; everything else keeps
    the reference's rounding).
  * per-cell tallies of a whole step: 1e-9 relative (the GPU adds deposits with
    atomics in a different order).
"""
import numpy as np
import pytest

from conftest import golden
from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, StormError
from storm_b200.units import UNITS

pytestmark = pytest.mark.gpu

REL = 1e-12


def close(a, b, rel=REL, atol=0.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + atol


def _replay(engine, oracle_lib, g):
    b = oracle_lib.ReplayBatch(g["before"], g["cell"], g["tape_offset"], g["tape_length"], g["tape"])
    engine.set_cell_physics(g["sigma_a"], np.zeros(engine.n), g["fleck"])
    engine.replay(b)
    return b


def _check_replay(b, g, ncells, near_tie_allowance=0.001, time_rel=0.0):
    n = len(g["cell"])
    st_ok = b["phys_status"] == g["status"]
    # a status flip is only acceptable on a near tie of two event times
    assert st_ok.mean() >= 1 - near_tie_allowance, (~st_ok).sum()
    ok = st_ok
    np.testing.assert_array_equal(b["draws_used"][ok], g["tape_length"][ok])
    moved = ok & (g["status"] == 1)
    np.testing.assert_array_equal(b["phys_next_cell"][moved].astype(np.int64), g["next"][moved])
    names = ["phys_x", "phys_y", "phys_z", "phys_vx", "phys_vy", "phys_vz", "phys_time_left", "phys_weight"]
    for k, nm in enumerate(names):
        if k < 3:
            atol = 1e-13                     # positions: cm, box size 1
        elif k == 7:
            # w *= 1 + expm1(-tau): for large tau the sum cancels, so an ulp of
            # CUDA's expm1 is an ulp of the segment's starting weight
            atol = 8e-16 * np.abs(g["before"][ok, 7])
        elif k == 6:
            # timeLeft - dt cancels when the event time is close to census
            atol = time_rel * np.abs(g["before"][ok, 6]) + 1e-300
        else:
            atol = 1e-300
        good = close(b[nm][ok], g["after"][ok, k], atol=atol)
        assert good.all(), (nm, np.where(~good)[0][:5])
    dm = g["tallies"][:, 1] - g["tallies"][:, 0]
    de = g["tallies"][:, 3] - g["tallies"][:, 2]
    scale_m = np.abs(g["tallies"][:, 1]) * 4e-16
    scale_e = np.abs(g["tallies"][:, 3]) * 4e-16
    assert (np.abs(b["dep_material"][ok] - dm[ok]) <= 1e-12 * np.abs(dm[ok]) + scale_m[ok] + 1e-300).all()
    assert (np.abs(b["dep_erad"][ok] - de[ok]) <= 1e-12 * np.abs(de[ok]) + scale_e[ok] + 1e-300).all()
    ch = ok & (g["next_cell"] >= 0)
    mgr = np.stack([b["mgr_x"], b["mgr_y"], b["mgr_z"], b["mgr_vx"], b["mgr_vy"], b["mgr_vz"]], 1)
    for k in range(6):
        assert close(mgr[ch, k], g["next_before"][ch, k], atol=1e-13 if k < 3 else 1e-300).all(), k
    np.testing.assert_array_equal(b["mgr_cell"][ch].astype(np.int64), g["next_cell"][ch])
    return (b["phys_status"] == g["status"]).sum(), n


def test_replay_reference_records_slab(oracle_lib):
    g = golden("replay_slab.npz")
    p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50)
    e = Engine(p)
    b = _replay(e, oracle_lib, g)
    same, n = _check_replay(b, g, p.ncells)
    assert same == n


def test_replay_reference_records_random_walk(oracle_lib):
    g = golden("replay_cube_rw.npz")
    p = problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20)
    e = Engine(p)
    b = _replay(e, oracle_lib, g)
    _check_replay(b, g, p.ncells)
    np.testing.assert_array_equal(b["used_random_walk"], g["used_rw"])


def test_random_walk_tables_and_samplers(oracle_lib):
    p = problems.step_cube(n=4)
    e = Engine(p)
    tau, surv, rad = e.rw_tables()
    otau, osurv, orad = oracle_lib.rw_tables()
    np.testing.assert_array_equal(tau, otau)        # host-built with the reference's arithmetic
    np.testing.assert_array_equal(surv, osurv)
    assert np.abs(rad - orad).max() < 1e-12           # device-built: CUDA exp/sin/cos/erf
    g = golden("rw_samples.npz")
    leak, radius = e.rw_sample(g["xi_leak"], g["tau"], g["xi_rad"])
    assert close(leak, g["leak"], 1e-12).all()
    assert (np.abs(radius - g["radius"]) < 1e-12).all()


def test_allocation_matches_reference():
    """Photon counts per cell: bit-exact against the reference's
    getLastSourcePhotonsPerCell, including cells whose share floors to 49."""
    g = golden("allocation_slab.npz")
    for s in range(len(g["photons"])):
        p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50)
        p.temperature = g["temperature"][s]
        p.internal_energy = g["internal_energy"][s]
        e = Engine(p)
        e.phase("begin")
        e.phase("prestep")
        c = e.cells()
        assert close(c["sigma_a"], g["sigma_a"][s], 1e-14).all()
        assert close(c["fleck"], g["fleck"][s], 1e-14).all()
        e.set_cell_physics(g["sigma_a"][s], np.zeros(p.ncells), g["fleck"][s])
        e.phase("emit")
        counts, _ = e.emission()
        np.testing.assert_array_equal(counts, g["photons"][s])


def _pair(p):
    from oracle import orc
    return Engine(p), orc.Oracle(p)


def _compare_census(ce, co):
    assert ce.n == co.n
    if ce.n == 0:
        return
    for f in ("x", "y", "z", "vx", "vy", "vz", "weight", "initial_weight"):
        ok = close(getattr(ce, f), getattr(co, f), 1e-12, atol=1e-300 if f[0] != "x" else 1e-14)
        assert ok.mean() > 0.999, (f, (~ok).sum())
    np.testing.assert_array_equal(ce.cell, co.cell)


@pytest.mark.parametrize("kind", ["slab", "cube"])
def test_full_step_matches_oracle(oracle_lib, kind):
    """One whole step on identical Philox streams: the GPU and the oracle follow
    the same histories, so counts agree exactly and tallies to rounding."""
    if kind == "slab":
        p = problems.gray_slab(new_photons_per_cell=5, face_packets=3000, comb_nmin=50)
        steps = 3
    else:
        p = problems.step_cube(n=12, new_photons_per_cell=3, face_packets=60, comb_nmin=10)
        steps = 2
    e, o = _pair(p)
    for s in range(steps):
        se = e.step()
        so = o.step()
        for k in ("emitted_cells", "emitted_faces", "census_out_pre_comb", "census_out", "segments", "escaped",
                  "cutoff", "rw_steps"):
            assert se[k] == so[k], (s, k, se[k], so[k])
        for k in ("energy_emitted", "energy_deposited", "energy_escaped", "energy_census_out"):
            assert close(se[k], so[k], 1e-9), (s, k)
        ce, co = e.cells(), o.cells()
        for k in ("temperature", "internal_energy", "erad_time_avg", "erad_census"):
            assert close(ce[k], co[k], 1e-9, atol=1e-300).all(), (s, k)
        np.testing.assert_array_equal(ce["segments"], co["segments"])
        _compare_census(e.census(), o.census())


def _balance(st):
    src = st["energy_census_in"] + st["energy_emitted"]
    sink = st["energy_deposited"] + st["energy_escaped"] + st["energy_census_pre_comb"]
    return abs(src - sink) / max(src, 1e-300)


def test_energy_conservation_step_cube():
    p = problems.step_cube(n=32, new_photons_per_cell=3, face_packets=200, comb_nmin=10)
    e = Engine(p)
    for _ in range(3):
        st = e.step()
        assert _balance(st) < 1e-10
        assert abs(st["energy_census_out"] - st["energy_census_pre_comb"]) <= 1e-10 * st["energy_census_pre_comb"]
        assert st["rw_steps"] > 0


def test_comb_matches_oracle(oracle_lib):
    """CombPopulationControl on the same census: the GPU (radix sort + per-cell
    comb) and the oracle produce the same particles in the same order."""
    from test_oracle import synthetic_census, _comb_invariants
    from oracle import ref
    p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=8, comb_factor=1.5)
    pre = synthetic_census(p, 3000, 3, ref.Particles)
    e = Engine(p)
    post = e.population_control(pre)
    _comb_invariants(pre, post, p)
    o = oracle_lib.Oracle(p)
    o.set_census(pre)
    o.phase("comb")
    oc = o.census()
    assert post.n == oc.n
    np.testing.assert_array_equal(post.cell, oc.cell)
    for f in ("x", "y", "z", "vx", "vy", "vz", "weight", "initial_weight"):
        np.testing.assert_array_equal(getattr(post, f), getattr(oc, f), err_msg=f)
    np.testing.assert_allclose(e.cells()["erad_census"], np.bincount(oc.cell, weights=oc.weight, minlength=p.ncells),
                               rtol=1e-15)


@pytest.mark.parametrize("crowd", [(600, 2000, 5000), (9000,)])
def test_comb_crowded_cells_match_oracle(oracle_lib, crowd):
    """Cells far above the mean population: runs of 513-8192 census particles
    are sorted by a block each, and a run above 8192 sends the whole comb to
    the radix-sort path.  Both give the oracle's particles in its order."""
    from test_oracle import synthetic_census
    from oracle import ref
    p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=8, comb_factor=1.5)
    n = 3000 + sum(crowd)
    pre = synthetic_census(p, n, 7, ref.Particles)
    at = 3000
    for c, k in zip((5, 40, 77), crowd):
        pre.cell[at:at + k] = c
        at += k
    xc, yc, zc = p.cell_centers()
    pre.x, pre.y, pre.z = xc[pre.cell].copy(), yc[pre.cell].copy(), zc[pre.cell].copy()
    e = Engine(p)
    post = e.population_control(pre)
    o = oracle_lib.Oracle(p)
    o.set_census(pre)
    o.phase("comb")
    oc = o.census()
    assert post.n == oc.n
    np.testing.assert_array_equal(post.cell, oc.cell)
    for f in ("x", "y", "z", "vx", "vy", "vz", "weight", "initial_weight"):
        np.testing.assert_array_equal(getattr(post, f), getattr(oc, f), err_msg=f)


def test_step_cube_statistics_vs_oracle(oracle_lib):
    """Several steps of the step-opacity cube on independent seeds: GPU and
    oracle agree cell by cell under the batch gate."""
    from batchcheck import assert_agree, run_batch

    def prob(s):
        return problems.step_cube(n=8, new_photons_per_cell=4, face_packets=80, comb_nmin=20, seed=s)
    assert_agree(run_batch(Engine, prob, range(10, 26), 4), run_batch(oracle_lib.Oracle, prob, range(50, 66), 4),
                 "step cube 8^3: engine vs oracle")


def test_errors_are_reported():
    p = problems.gray_slab()
    p.precision = 7   # no such precision
    with pytest.raises(StormError):
        Engine(p)
    e = Engine(problems.gray_slab())
    from storm_b200.engine import Particles
    bad = Particles(1)
    bad.cell[:] = 10 ** 6
    with pytest.raises(StormError):
        e.set_census(bad)


@pytest.mark.parametrize("precision", [A.PRECISION_FP64, A.PRECISION_FP32_TRACK])
def test_census_without_step_fields_steps_the_same(precision):
    """storm_cuda_set_census with time_left and initial_weight left out (the
    step sets both for every census particle) steps exactly like the full
    census: same counts, temperatures to the atomics' summation order."""
    p = problems.step_cube(n=10, new_photons_per_cell=3, face_packets=60, comb_nmin=10, precision=precision)
    src = Engine(p)
    src.step()
    census = src.census()
    src.close()
    full, lean = Engine(p), Engine(p)
    full.set_census(census)
    lean.set_census(census, step_fields=False)
    lc = lean.census()
    assert (lc.time_left == 0).all() and (lc.initial_weight == 0).all()
    sf, sl = full.step(), lean.step()
    for k in ("census_in", "emitted_cells", "census_out", "segments", "escaped", "cutoff"):
        assert sf[k] == sl[k], k
    assert close(full.cells()["temperature"], lean.cells()["temperature"], 1e-9).all()
    full.close()
    lean.close()
