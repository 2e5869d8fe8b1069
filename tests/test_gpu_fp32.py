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
    """Per-cell material temperature after several steps: the FP32-tracking and
    FP64 forms agree within the seed-to-seed statistical error."""
    def run(precision, seeds):
        out = []
        for s in seeds:
            p = problems.step_cube(n=16, new_photons_per_cell=4, face_packets=120, comb_nmin=20, seed=s,
                                   precision=precision)
            e = Engine(p)
            for _ in range(4):
                e.step()
            out.append(e.cells()["temperature"])
        return np.array(out)
    seeds = range(300, 308)
    a = run(A.PRECISION_FP64, seeds)
    b = run(A.PRECISION_FP32_TRACK, seeds)
    ma, mb = a.mean(0), b.mean(0)
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    hot = ma > 1.5 * a.min()
    z = np.abs(ma - mb)[hot] / np.maximum(se[hot], 1e-12 * ma[hot])
    assert hot.sum() > 100
    assert (z < 3.0).mean() > 0.97, (z > 3).sum()
    assert z.mean() < 1.2
