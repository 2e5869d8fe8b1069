"""The FP32-tracking form: cell index + FP32 cell-local offset, FP32 direction
and distances; time, weights, deposits and tallies in FP64.

Acceptance: energy is conserved per step to 1e-10 relative (deposit and weight
update share one attenuation factor), and per-cell results agree with the FP64
form within the statistical error estimated from independent seeds.
"""
import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, Particles
from storm_b200.units import UNITS

pytestmark = pytest.mark.gpu


def _balance(st):
    src = st["energy_census_in"] + st["energy_emitted"]
    sink = st["energy_deposited"] + st["energy_escaped"] + st["energy_census_pre_comb"]
    return abs(src - sink) / max(src, 1e-300)


@pytest.mark.parametrize("kind", ["slab", "cube"])
def test_fp32_energy_conservation(kind):
    if kind == "slab":
        p = problems.gray_slab(new_photons_per_cell=5, face_packets=3000, comb_nmin=50, precision=A.PRECISION_FP32_TRACK)
    else:
        p = problems.step_cube(n=24, new_photons_per_cell=3, face_packets=100, comb_nmin=10,
                               precision=A.PRECISION_FP32_TRACK)
    e = Engine(p)
    for _ in range(4):
        st = e.step()
        assert _balance(st) < 1e-10, st
        assert abs(st["energy_census_out"] - st["energy_census_pre_comb"]) <= 1e-10 * max(st["energy_census_pre_comb"], 1e-300)
    c = e.census()
    # every census particle lies inside its own cell
    xe, ye, ze = p.x_edges, p.y_edges, p.z_edges
    nx, ny, nz = p.shape
    i, j, k = c.cell % nx, (c.cell // nx) % ny, c.cell // (nx * ny)
    assert ((c.x >= xe[i]) & (c.x <= xe[i + 1]) & (c.y >= ye[j]) & (c.y <= ye[j + 1]) & (c.z >= ze[k]) &
            (c.z <= ze[k + 1])).all()


def test_fp32_census_round_trip():
    p = problems.step_cube(n=8, precision=A.PRECISION_FP32_TRACK)
    e = Engine(p)
    rng = np.random.default_rng(3)
    n = 1000
    q = Particles(n)
    q.cell = rng.integers(0, p.ncells, n).astype(np.uint32)
    xc, yc, zc = p.cell_centers()
    h = 0.5 / 8
    q.x = xc[q.cell] + rng.uniform(-h, h, n)
    q.y = yc[q.cell] + rng.uniform(-h, h, n)
    q.z = zc[q.cell] + rng.uniform(-h, h, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    q.vx, q.vy, q.vz = (d * 2.99792458e10).T
    q.weight = rng.random(n) + 0.5
    q.initial_weight = q.weight.copy()
    e.set_census(q)
    back = e.census()
    np.testing.assert_array_equal(back.cell, q.cell)
    assert np.abs(back.x - q.x).max() < 1e-7 * h * 4
    assert np.abs(back.vx - q.vx).max() < 1e-6 * 2.99792458e10
    np.testing.assert_array_equal(back.weight, q.weight)


def test_fp32_agrees_with_fp64_within_statistics():
    """Per cell after several steps (material temperature, deposit, radiation
    energies): the FP32-tracking and FP64 forms, on independent seeds, agree
    under the batch gate."""
    from batchcheck import assert_agree, run_batch

    def prob(precision):
        return lambda s: problems.step_cube(n=16, new_photons_per_cell=4, face_packets=120, comb_nmin=20, seed=s,
                                            precision=precision)
    res = assert_agree(run_batch(Engine, prob(A.PRECISION_FP64), range(300, 316), 4),
                       run_batch(Engine, prob(A.PRECISION_FP32_TRACK), range(400, 416), 4),
                       "step cube 16^3: FP32 vs FP64")
    assert res["temperature"]["tests"] > 100


def test_fp32_emission_follows_fp64_draws():
    """Cell and face source packets of the FP32 form: drawn in the cell's own
    FP32 frame from the same Philox draws as the FP64 form, so each packet sits
    where the FP64 packet sits to FP32 rounding (the tetrahedron pick may differ
    when 12 u lands within FP32 rounding of an integer)."""
    p = problems.step_cube(n=16, new_photons_per_cell=5, face_packets=40, comb_nmin=10)
    dt = p.dt
    banks = []
    for prec in (A.PRECISION_FP64, A.PRECISION_FP32_TRACK):
        q = problems.step_cube(n=16, new_photons_per_cell=5, face_packets=40, comb_nmin=10)
        q.precision = prec
        e = Engine(q)
        for ph in ("begin", "prestep", "emit"):
            e.phase(ph, dt)
        banks.append(e.bank())
        e.close()
    b64, b32 = banks
    assert b64.n == b32.n > 0
    np.testing.assert_array_equal(b64.cell, b32.cell)
    np.testing.assert_array_equal(b64.id, b32.id)
    np.testing.assert_array_equal(b64.time_left, b32.time_left)
    np.testing.assert_array_equal(b64.weight, b32.weight)
    h = 0.5 / 16
    dpos = np.max(np.abs(np.stack([b64.x - b32.x, b64.y - b32.y, b64.z - b32.z])), axis=0)
    assert (dpos <= 1e-6 * h).mean() > 0.999, np.sort(dpos)[-5:]
    assert (dpos <= 2 * h).all()
    c = UNITS["clight"]
    # 2^-23 quantisation of cos(theta) moves the direction by ~1e-7 / sin(theta)
    ddir = np.max(np.abs(np.stack([b64.vx - b32.vx, b64.vy - b32.vy, b64.vz - b32.vz]) / c), axis=0)
    assert (ddir <= 1e-4).mean() > 0.999, np.sort(ddir)[-5:]
