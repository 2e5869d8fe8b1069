"""The polyhedral RandomInCellPositionSampler restated in tests/polysample.py
(the two-pass volume sum that the GPU emission's tetrahedron table is tested
against) equals the reference's own sampler bit for bit, from the uniforms the
reference drew, on a Voronoi mesh through the grid stand-in's polyhedral mode."""
import numpy as np
import pytest

from polysample import two_pass_point
from storm_b200 import problems
from storm_b200.mesh import build_voronoi


def test_two_pass_restatement_matches_the_reference_sampler(ref_lib):
    mesh = build_voronoi(np.random.default_rng(7).random((40, 3)) * 0.98 + 0.01)
    p = problems.voronoi_cube(ncells=40, packets_per_step=4e3, seed=11, mesh=mesh)
    r = ref_lib.Reference(p)
    cells = np.repeat(np.arange(mesh.ncells, dtype=np.uint32), 25)
    pos, tape, nd = r.sample_in_cell(cells, 5)
    r.close()
    assert (nd == 4).all(), np.unique(nd)
    u = tape.reshape(-1, 4)
    for k, c in enumerate(cells):
        assert tuple(pos[k]) == two_pass_point(mesh, int(c), u[k]), (k, int(c))
