"""Checkpoint and restore of a handle's step-to-step state (census bank, cell
state, face temperatures, step counter): a run interrupted after two steps and
resumed from its checkpoint in a fresh handle repeats the uninterrupted run.
Tallies are summed with atomics, so temperatures agree to 1e-9 rather than bit
for bit."""
import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, StormError

pytestmark = pytest.mark.gpu

CASES = {
    "cube_fp64": lambda: problems.step_cube(n=16, new_photons_per_cell=3, face_packets=60, comb_nmin=10),
    "cube_fp32": lambda: problems.step_cube(n=16, new_photons_per_cell=3, face_packets=60, comb_nmin=10,
                                            precision=A.PRECISION_FP32_TRACK),
    "mg_fp32": lambda: problems.mg_cube(n=6, groups=64, kappa0=1.0, new_photons_per_cell=4, comb_nmin=4,
                                        precision=A.PRECISION_FP32_TRACK),
    "voronoi_fp64": lambda: problems.voronoi_cube(ncells=300, packets_per_step=2e4, seed=3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_resume_from_checkpoint_repeats_the_run(name):
    p = CASES[name]()
    a = Engine(p)
    for _ in range(4):
        a.step()
    Ta, na = a.cells()["temperature"], a.census_count()
    a.close()
    b = Engine(p)
    for _ in range(2):
        b.step()
    blob = b.checkpoint()
    b.close()
    c = Engine(p)
    c.restore(blob)
    for _ in range(2):
        c.step()
    Tc, nc = c.cells()["temperature"], c.census_count()
    assert abs(int(nc) - int(na)) <= 1e-3 * na
    np.testing.assert_allclose(Tc, Ta, rtol=1e-9)
    c.close()


def test_checkpoint_rejects_another_problem():
    a = Engine(problems.step_cube(n=8))
    a.step()
    blob = a.checkpoint()
    a.close()
    other = Engine(problems.step_cube(n=10))
    with pytest.raises(StormError):
        other.restore(blob)
    with pytest.raises(StormError):
        other.restore(blob[:40])
    other.close()


def test_rejected_checkpoint_leaves_the_handle_unchanged():
    """A checkpoint whose census names a cell outside the grid, or whose header
    claims more particles than the buffer holds, is refused before any of the
    handle's state is overwritten: the handle keeps its census and cell state
    and steps on as if nothing had been loaded."""
    import struct
    p = problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=10)
    a = Engine(p)
    a.step()
    blob = bytearray(a.checkpoint())
    a.step()
    T0, n0 = a.cells()["temperature"], a.census_count()
    head = 8 + 4 * 4   # magic, abi, precision, groups, ncells
    n = struct.unpack_from("<Q", blob, head)[0]
    assert n > 0
    bad_cell = bytearray(blob)
    cell_at = 88 + 9 * 8 * n        # header (88 bytes), then nine 8-byte arrays, then the cell ids
    struct.pack_into("<I", bad_cell, cell_at + 4 * (n // 2), p.ncells + 5)
    huge = bytearray(blob)
    struct.pack_into("<Q", huge, head, 1 << 62)
    for b in (bad_cell, huge):
        with pytest.raises(StormError):
            a.restore(bytes(b))
        assert a.census_count() == n0
        np.testing.assert_array_equal(a.cells()["temperature"], T0)
    a.step()
    assert a.census_count() > 0
    a.close()
