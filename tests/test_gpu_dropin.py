"""MonteCarloManagerCUDA (include/storm/MonteCarloManagerCUDA.hpp), the C++
drop-in for MonteCarloManagerSerial, compiled against the reference's own grid,
cells, RadiationIMC, comb and boundary objects (oracle/_ref/libstormdropin.so).

* test_dropin_matches_engine: the template converts the reference's
  std::vector<Particle> and cell vectors to the C ABI and back every step; the
  result must equal the Python binding driving the same engine with the same
  per-step uploads (same Philox streams): counts exact, floats to 1e-12.
* test_dropin_vs_serial_manager: the drop-in and the reference's serial manager
  on the same problem, independent seeds: per-cell temperature, deposit and
  radiation energies under the batch gate of storm_b200.batchstats.
Both run gray problems and a 30-group multigroup problem (RadiationIMC<..., 30>,
census frequencies carried through the template).
* test_dropin_lowers_stock_boundaries: VacuumBoundary, RigidBoundary,
  SideTemperature and TwoSidesTemperature are recognised by type; their
  first-step emission per cell (GetBeginningParticleCount) equals the serial
  manager's with the same boundary object type.
* test_dropin_slab_with_plugin_opacity_matches_reference_batch: the 100-cell
  slab for all 100 steps through the template, with TwoSidesTemperature
  lowered by type and the temperature-dependent opacity kappa = 10 T^-3
  evaluated through the opacity plug-in before every step, against the
  reference's 32-seed batch.
"""
import ctypes as C
import os

import numpy as np
import pytest

from storm_b200 import batchstats
from storm_b200 import problems
from storm_b200 import _abi as A
from storm_b200.engine import Engine

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "libstormdropin.so")


def _lib():
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in harness (oracle/_ref/libstormdropin.so) not built")
    from oracle import ref
    L = C.CDLL(DROPIN)
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    L.dropin_create.restype = vp
    L.dropin_create.argtypes = [C.POINTER(A.StormProblemDesc), C.c_int, C.c_char_p, C.c_size_t]
    L.dropin_create_plugins.restype = vp
    L.dropin_create_plugins.argtypes = [C.POINTER(A.StormProblemDesc), C.c_int, C.c_int, C.c_int, C.c_char_p,
                                        C.c_size_t]
    L.dropin_beginning_counts.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.ref_beginning_counts.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.ref_get_motion.argtypes = [vp, dp, dp]
    L.dropin_destroy.argtypes = [vp]
    L.dropin_ref.restype = vp
    L.dropin_ref.argtypes = [vp]
    L.dropin_last_error.restype = C.c_char_p
    L.dropin_last_error.argtypes = [vp]
    L.dropin_step.argtypes = [vp, C.c_double, C.POINTER(ref.RefStepOut)]
    L.dropin_get_cells.argtypes = [vp, dp, dp, dp, C.POINTER(C.c_uint64)]
    L.ref_get_cells.argtypes = [vp] + [dp] * 6 + [C.POINTER(C.c_uint64)]
    L.ref_census_count.restype = C.c_uint64
    L.ref_census_count.argtypes = [vp]
    L.ref_get_census.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
    return L


class DropIn:
    """One reference problem whose manager is MonteCarloManagerCUDA."""

    def __init__(self, L, problem, precision=0, boundary_kind=0, opacity_from_plugin=False):
        self.L, self.problem = L, problem
        self.desc = problem.to_desc()
        err = C.create_string_buffer(512)
        self.h = L.dropin_create_plugins(C.byref(self.desc), precision, boundary_kind, int(opacity_from_plugin),
                                         err, 512)
        if not self.h:
            raise RuntimeError("dropin_create failed: " + err.value.decode())
        self.ref = L.dropin_ref(self.h)
        self.n = problem.ncells

    def close(self):
        if self.h:
            self.L.dropin_destroy(self.h)
            self.h = None

    def step(self):
        from oracle import ref
        out = ref.RefStepOut()
        if self.L.dropin_step(self.h, self.problem.dt, C.byref(out)) != 0:
            raise RuntimeError(self.L.dropin_last_error(self.h).decode())
        return out.as_dict()

    def cells(self):
        keys = ("temperature", "internal_energy", "erad_time_avg", "erad_census", "sigma_a", "fleck")
        out = {k: np.zeros(self.n) for k in keys}
        segs = np.zeros(self.n, np.uint64)
        self.L.ref_get_cells(self.ref, *[A.ptr(out[k]) for k in keys], A.ptr(segs, C.c_uint64))
        # the serial manager's RadiationIMC did not run: time-averaged Erad,
        # opacities, Fleck factors and segment counters come from the drop-in's getters
        self.L.dropin_get_cells(self.h, A.ptr(out["erad_time_avg"]), A.ptr(out["sigma_a"]), A.ptr(out["fleck"]),
                                A.ptr(segs, C.c_uint64))
        out["segments"] = segs
        return out

    def beginning_counts(self):
        out = np.zeros(self.n, np.uint64)
        assert self.L.dropin_beginning_counts(self.h, A.ptr(out, C.c_uint64)) == 0
        return out

    def census(self):
        from oracle import ref
        n = self.L.ref_census_count(self.ref)
        p = ref.Particles(n)
        s = p.soa()
        self.L.ref_get_census(self.ref, C.byref(s))
        return p


def _close(a, b, rel, atol=1e-300):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + atol


@pytest.mark.parametrize("kind", ["slab", "cube", "multigroup", "stratified", "ddmc", "voronoi", "hydro"])
def test_dropin_matches_engine(kind):
    L = _lib()
    if kind == "slab":
        p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50)
    elif kind == "cube":
        p = problems.step_cube(n=12, new_photons_per_cell=3, face_packets=60, comb_nmin=10)
    elif kind == "multigroup":   # RadiationIMC<..., 30> with multigroup opacity and a Planck face source
        p = problems.densmore2012(nx=16, new_photons_per_cell=4, boundary_per_face=50)
        p.comb_nmin = 10
    elif kind == "stratified":   # StratifiedCombPopulationControl with frequency bins
        p = problems.strat_cube(n=4)
    elif kind == "voronoi":   # a Voronoi grid, lowered by the template through the Grid API
        p = problems.voronoi_cube(ncells=200, packets_per_step=1e4, seed=3)
    elif kind == "hydro":   # moving cells: velocities in and momenta out through the cell and extensives types
        import sys
        from conftest import GOLDEN
        sys.path.insert(0, GOLDEN)
        import make_golden as MG
        p = problems.step_cube(n=10, new_photons_per_cell=3, face_packets=60, comb_nmin=10)
        p.with_hydro = True
        p.cell_velocity = MG.hydro_velocity(p)
    else:   # DDMC leakage in the thick half
        p = problems.ddmc_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=10)
    d = DropIn(L, p)
    e = Engine(p)
    try:
        for s in range(3):
            # the drop-in uploads the caller's cells and census every step
            ce = e.cells()
            e.set_cell_state(ce["temperature"], ce["internal_energy"], ce["internal_energy"])
            e.set_census(e.census())
            if p.with_hydro:
                e.set_cell_motion(*e.cell_motion())
            se = e.step()
            sd = d.step()
            if p.with_hydro:
                vd, md = np.zeros((p.ncells, 3)), np.zeros((p.ncells, 3))
                L.ref_get_motion(d.ref, A.ptr(vd), A.ptr(md))
                ve, me = e.cell_motion()
                assert _close(vd, ve, 1e-12, atol=1e-3).all() and _close(md, me, 1e-12, atol=1e-9).all(), s
            assert sd["initial"] == se["census_in"]
            assert sd["prestep"] == se["emitted_cells"] + se["emitted_faces"]
            assert sd["end"] == se["census_out"]
            assert sd["segments"] == se["segments"]
            cd, ce = d.cells(), e.cells()
            for k in ("temperature", "internal_energy", "erad_time_avg", "erad_census", "sigma_a", "fleck"):
                assert _close(cd[k], ce[k], 1e-12).all(), (s, k)
            np.testing.assert_array_equal(cd["segments"], ce["segments"])
            # tallies are summed with atomics, so material temperatures (and with
            # them Fleck factors and collision distances) may differ in the last
            # bit between the two runs: census floats compare to 1e-12
            pd, pe = d.census(), e.census()
            assert pd.n == pe.n
            np.testing.assert_array_equal(pd.cell, pe.cell)
            fields = ["x", "y", "z", "vx", "vy", "vz", "time_left", "weight", "initial_weight"]
            if p.groups:
                fields.append("frequency")
            for f in fields if pd.n else ():
                ok = _close(getattr(pd, f), getattr(pe, f), 1e-12, atol=1e-15 if f in "xyz" else 1e-300)
                assert ok.mean() > 0.999, (s, f, (~ok).sum())
    finally:
        d.close()
        e.close()


@pytest.mark.parametrize("kind", ["cube", "multigroup"])
def test_dropin_vs_serial_manager(kind):
    L = _lib()
    from oracle import ref

    def make_problem(s):
        if kind == "cube":
            return problems.step_cube(n=8, new_photons_per_cell=4, face_packets=80, comb_nmin=20, seed=s)
        p = problems.densmore2012(nx=24, new_photons_per_cell=6, boundary_per_face=200, seed=s)
        p.comb_nmin = 20
        return p

    steps = 4 if kind == "cube" else 12

    def run(make, seeds):
        out = []
        for s in seeds:
            p = make_problem(s)
            m = make(p)
            out.append(batchstats.run_snapshots(m, p, steps, (steps,)))
            m.close()
        return np.array(out)

    a = run(lambda p: DropIn(L, p), range(10, 22))
    b = run(lambda p: ref.Reference(p), range(50, 62))
    res = batchstats.compare(a, b)
    print(kind, res["all"], res["totals"])
    assert res["all"]["tests"] > 0 and res["passed"], res["all"] | {"totals": res["totals"]}


@pytest.mark.parametrize("kind", ["rigid", "vacuum", "side", "two_sides"])
def test_dropin_lowers_stock_boundaries(kind):
    """The stock boundary objects lowered by type: the first step's particles
    per cell when transport begins (emission only; GetBeginningParticleCount)
    equal the serial manager's with the same boundary type, and a few steps run.
    TwoSidesTemperature at T_R = 0 emits zero-weight packets at x-high in the
    reference and none on the device, so its last cell is left out."""
    L = _lib()
    from oracle import ref
    bk = {"rigid": ref.BOUNDARY_RIGID, "vacuum": ref.BOUNDARY_VACUUM, "side": ref.BOUNDARY_SIDE_TEMPERATURE,
          "two_sides": ref.BOUNDARY_TWO_SIDES_TEMPERATURE}[kind]
    p = problems.gray_slab(nx=20, new_photons_per_cell=20, face_packets=3000, comb_nmin=50)
    d = DropIn(L, p, boundary_kind=bk, opacity_from_plugin=True)
    r = ref.Reference(p, boundary_kind=bk)
    try:
        d.step()
        r.step()
        cd = d.beginning_counts()
        cr = np.zeros(p.ncells, np.uint64)
        assert L.ref_beginning_counts(C.c_void_p(r.h), A.ptr(cr, C.c_uint64)) == 0
        keep = slice(0, p.ncells - 1) if kind == "two_sides" else slice(None)
        np.testing.assert_array_equal(cd[keep], cr[keep])
        if kind in ("side", "two_sides"):
            assert cd[0] > cd[1]   # the hot face's packets start in the first cell
        for _ in range(3):
            d.step()
        c = d.cells()
        assert np.isfinite(c["temperature"]).all() and (c["temperature"] > 0).all()
    finally:
        d.close()
        r.close()


def test_dropin_slab_with_plugin_opacity_matches_reference_batch():
    """The 100x1x1 slab (1 keV at x=0, vacuum at x=1, reflecting y/z,
    kappa = min(10 T_keV^-3, 1e6)) for all 100 steps through
    MonteCarloManagerCUDA: TwoSidesTemperature(1 keV, 0) lowered by type, the
    opacity evaluated through the reference-side opacity plug-in on the
    caller's cells before every step (CELL_TABLE callbacks), 24 seeds against
    the reference serial path's 32 (tests/golden/reference_batch.npz, c1)
    under the batch gate."""
    import json
    import sys
    from conftest import GOLDEN, golden
    from oracle import ref
    sys.path.insert(0, GOLDEN)
    import make_reference_batch as MB
    w = MB.WORKLOADS["c1"]
    L = _lib()
    runs = []
    for s in range(3000, 3024):
        p = MB.workload("c1", s)
        d = DropIn(L, p, boundary_kind=ref.BOUNDARY_TWO_SIDES_TEMPERATURE, opacity_from_plugin=True)
        runs.append(batchstats.run_snapshots(d, p, w["steps"], w["snapshots"]))
        d.close()
    g = golden("reference_batch.npz")
    fx = {k[3:]: v for k, v in g.items() if k.startswith("c1_")}
    res = batchstats.compare(np.array(runs), fx)
    print(json.dumps({"workload": "c1 through MonteCarloManagerCUDA", "all": res["all"], "totals": res["totals"]}))
    assert res["all"]["tests"] > 0.1 * fx["mean"].size   # cold cells carry no sampling noise
    assert res["passed"], res["all"] | {"totals": res["totals"]}


def test_dropin_fp32_tracking_runs():
    """The FP32-tracking form behind the same template: census and material
    energy stay finite and the step conserves the census count bounds."""
    L = _lib()
    p = problems.step_cube(n=12, new_photons_per_cell=3, face_packets=60, comb_nmin=10)
    d = DropIn(L, p, precision=1)
    try:
        for _ in range(3):
            st = d.step()
            assert st["end"] > 0
        c = d.cells()
        assert np.isfinite(c["temperature"]).all() and (c["temperature"] > 0).all()
        pc = d.census()
        assert np.isfinite(pc.weight).all() and (pc.weight > 0).all()
    finally:
        d.close()
