"""storm_cuda_step_host (the census in from the host, the step, the new census
back, with the upload overlapped) against the same step as
storm_cuda_set_census + storm_cuda_step + storm_cuda_get_census from one
checkpoint: the same census bit for bit (each particle draws from its own
stream and the comb orders the census by key) and the same cell state to the
order of the FP64 tally sums; a census cell outside the mesh is refused before
the step changes the cell state."""
import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, Particles, StormError

pytestmark = pytest.mark.gpu

CASES = {
    "cube_fp32": lambda: problems.step_cube(n=16, new_photons_per_cell=3, face_packets=60, comb_nmin=10,
                                            precision=A.PRECISION_FP32_TRACK),
    "cube_fp64": lambda: problems.step_cube(n=16, new_photons_per_cell=3, face_packets=60, comb_nmin=10),
    "mg_fp32": lambda: problems.mg_cube(n=6, groups=64, kappa0=1.0, new_photons_per_cell=4, comb_nmin=4,
                                        precision=A.PRECISION_FP32_TRACK),
    "voronoi_fp32": lambda: problems.voronoi_cube(ncells=300, packets_per_step=2e4, seed=3,
                                                  precision=A.PRECISION_FP32_TRACK),
}
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "weight", "cell")


def _arrays(p, with_nu):
    out = {f: np.array(getattr(p, f)) for f in FIELDS}
    if with_nu:
        out["frequency"] = np.array(p.frequency)
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_step_host_equals_the_three_calls(name):
    p = CASES[name]()
    mg = p.groups >= 2
    e = Engine(p)
    e.step()   # from an empty census: the next step's pids reach further (a wider comb key)
    blob = e.checkpoint()
    host = e.census()
    n = host.n
    assert n > 0
    inbuf = Particles.pinned(n)
    for f in FIELDS + ("time_left", "initial_weight"):
        getattr(inbuf, f)[:n] = getattr(host, f)
    if mg:
        inbuf.frequency = np.array(host.frequency)
    outbuf = Particles.pinned(4 * n + 4096)
    if mg:
        outbuf.frequency = np.zeros(outbuf.n)
    st1, out1 = e.step_host(inbuf.view(n), outbuf)
    a1 = _arrays(out1, mg)
    T1 = e.cells()["temperature"]
    e.restore(blob)
    e.set_census(host, step_fields=False)
    st2 = e.step()
    out2 = e.census()
    a2 = _arrays(out2, mg)
    T2 = e.cells()["temperature"]
    e.close()
    for k in ("segments", "census_out", "census_out_pre_comb", "emitted_cells", "emitted_faces", "escaped"):
        assert st1[k] == st2[k], k
    for f, v in a2.items():
        assert np.array_equal(a1[f], v), f
    np.testing.assert_allclose(T1, T2, rtol=1e-12)


def test_step_host_refuses_a_census_cell_outside_the_mesh():
    p = CASES["cube_fp32"]()
    e = Engine(p)
    e.step()
    host = e.census()
    n = host.n
    bad = Particles.pinned(n)
    for f in FIELDS + ("time_left", "initial_weight"):
        getattr(bad, f)[:n] = getattr(host, f)
    bad.cell[n // 2] = p.ncells + 3
    T0 = e.cells()["temperature"].copy()
    out = Particles.pinned(4 * n + 4096)
    with pytest.raises(StormError):
        e.step_host(bad.view(n), out)
    assert e.census_count() == 0
    assert np.array_equal(e.cells()["temperature"], T0)
    st, out1 = e.step_host(host, out)   # the handle steps on
    assert st["segments"] > 0 and out1.n == e.census_count()
    e.close()


def test_step_host_with_reproducible_tallies_takes_the_three_calls():
    p = problems.step_cube(n=12, new_photons_per_cell=3, face_packets=60, comb_nmin=10,
                           precision=A.PRECISION_FP32_TRACK)
    p.reproducible_tallies = True
    a, b = Engine(p), Engine(p)
    a.step()
    b.step()
    ha, hb = a.census(), b.census()
    st1, out1 = a.step_host(ha, Particles(4 * ha.n + 4096))
    b.set_census(hb, step_fields=False)
    st2 = b.step()
    out2 = b.census()
    for f in FIELDS:
        assert np.array_equal(getattr(out1, f), getattr(out2, f)), f
    assert np.array_equal(a.cells()["temperature"], b.cells()["temperature"])
    a.close()
    b.close()
