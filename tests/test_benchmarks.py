"""The reference's full-run benchmark problems on the CPU: the problem
builders against the example sources' set-up, the time-step schedule, the L1
measures against known answers, and a short Densmore run through the
reference build (30 groups, multigroup face source)."""
import numpy as np
import pytest

from conftest import golden
from storm_b200 import _abi as A
from storm_b200 import benchmarks as B
from storm_b200 import problems as P
from storm_b200.units import UNITS

KEV_K = UNITS["kev_kelvin"]


def test_reference_curves_fixture():
    g = golden("reference_curves.npz")
    for k in range(1, 5):
        c = g[f"marshak_wave_{k}"]
        assert c.shape == (512, 3) and (np.diff(c[:, 0]) > 0).all()
    d = g["densmore2012"]
    assert d.shape[1] == 2 and d[0, 0] == 0.0 and 0.5 < d[0, 1] < 1.0


def test_marshak_l1_known_answers():
    ref = golden("reference_curves.npz")["marshak_wave_1"]
    x, t = ref[:, 0], ref[:, 1]
    assert B.marshak_l1(x, t, ref) < 1e-15
    # 10 % hotter everywhere: every compared point contributes 0.1
    assert B.marshak_l1(x, 1.1 * t, ref) == pytest.approx(0.1, rel=1e-12)
    # points at or below 1e-4 keV are not compared
    cold = ref.copy()
    cold[:, 1] = 0.5e-4 * KEV_K
    assert B.marshak_l1(x, t, cold) == -1.0


def test_densmore_l1_known_answer():
    ref = golden("reference_curves.npz")["densmore2012"]
    x = np.linspace(0.0, 3.0, 301)
    flat = np.full_like(x, 0.5 * KEV_K)
    assert B.densmore_l1(x, flat, ref) == pytest.approx(np.mean(np.abs(0.5 - ref[:, 1])), rel=1e-12)
    # reference points past the last simulated interval are skipped
    assert B.densmore_l1(x[:201], flat[:201], ref) == pytest.approx(
        np.mean(np.abs(0.5 - ref[ref[:, 0] <= 2.0, 1])), rel=1e-12)


def test_marshak_schedule():
    """The example's dt rule: 1000 steps of the initial dt, then dt = t/1000,
    the last step clipped to end at 1 ns."""
    for k in (1, 4):
        sched = list(B.marshak_schedule(k))
        dt0 = P.MARSHAK_PARAMS[k]["initial_dt"]
        assert sched[0] == (dt0, dt0)
        t = 0.0
        for t_now, dt in sched:
            assert t_now == max(t, dt0)
            t += dt
        assert t >= P.MARSHAK_FINAL_TIME and t - sched[-1][1] < P.MARSHAK_FINAL_TIME
        assert all(dt <= 5e-11 for _, dt in sched)


def test_marshak_problems_match_example_setup():
    p = P.marshak_wave(1)
    assert p.shape == (256, 1, 1) and p.x_edges[-1] == 0.2 and p.y_edges[-1] == 0.2 / 256
    assert p.faces[0].action == A.FACE_ESCAPE and p.faces[0].packets_per_face == 100
    assert all(f.action == A.FACE_REFLECT for f in p.faces[1:])
    assert (p.comb_nmin, p.comb_factor, p.new_photons_per_cell) == (15, 6.0, 15)
    # e_vol = f T^4 at T0 = 1 eV for problem 1 (rho = 1)
    f = 6.860085e14 / KEV_K ** 4
    assert np.allclose(p.internal_energy / p.volumes(), f * (1e-3 * KEV_K) ** 4, rtol=1e-14)
    p4 = P.marshak_wave(4)
    assert p4.shape == (512, 1, 1) and p4.x_edges[0] == 1e-5 and p4.x_edges[-1] == 1.0 + 1e-5
    w = np.diff(p4.x_edges)[:-1]
    assert np.allclose(w[1:] / w[:-1], 1.0096903847403653, rtol=1e-9)
    xc, _, _ = p4.cell_centers()
    assert np.allclose(p4.density_factor, np.power(xc, -40.0 / 139.0 * 1.9), rtol=1e-12)
    p3 = P.marshak_wave(3)
    assert p3.faces[0].source_temperature == pytest.approx(1.0470478 * (1e-6) ** (86.0 / 57.0) * KEV_K)


def test_densmore_problem_matches_example_setup():
    p = P.densmore2012()
    kev = UNITS["kev"]
    assert p.shape == (512, 1, 1) and p.groups == 30
    b = p.group_bounds
    assert b[0] == kev * 1e-4 and b[-1] == pytest.approx(kev * 1e2, rel=1e-12)
    assert np.allclose(b[1:] / b[:-1], (1e6) ** (1 / 30), rtol=1e-13)
    xc, _, _ = p.cell_centers()
    assert (p.sigma_a[xc < 2] == 10 * kev ** 3.5).all() and (p.sigma_a[xc >= 2] == 1000 * kev ** 3.5).all()
    assert (p.mg_p, p.mg_q, p.mg_s, p.mg_group_constant) == (3.0, 0.5, 0.0, False)
    assert p.temperature[0] == KEV_K / 1000 and p.faces[0].source_temperature == KEV_K
    assert (p.comb_nmin, p.comb_factor, p.dt) == (200, 5.0, 5e-12)


def test_densmore_reference_build_short_run(ref_lib):
    """Ten steps of a small Densmore slab through the reference build: energy
    is conserved, the census carries frequencies inside the group range, and
    the slab heats from the driven face."""
    p = P.densmore2012(nx=32, new_photons_per_cell=4, boundary_per_face=50)
    r = ref_lib.Reference(p)
    for _ in range(10):
        r.step(p.dt)
    c = r.census()
    assert (c.frequency >= p.group_bounds[0]).all() and (c.frequency <= p.group_bounds[-1]).all()
    T = r.cells()["temperature"]
    assert T[0] > T[-1] and T[0] > 2 * p.temperature[0]
    r.close()
