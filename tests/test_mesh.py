"""The Voronoi mesh builder (storm_mesh_voronoi, host code): the cells tile
the box, every cell is a closed polyhedron whose faces give back its volume
through the divergence theorem, interior faces lie on the bisector of their two
generators, and the build is deterministic."""
import numpy as np
import pytest

from storm_b200.mesh import build_voronoi


@pytest.fixture(scope="module")
def mesh_and_points():
    pts = np.random.default_rng(17).random((600, 3)) * (1 - 2e-9) + 1e-9
    return build_voronoi(pts), pts


def _outward(m, c, f):
    """Face f's unit normal pointing out of cell c (away from c's generator)."""
    n = m.face_normal[f] / np.linalg.norm(m.face_normal[f])
    return n if np.dot(m.face_cm[f] - m.points[c], n) > 0 else -n


def test_cells_tile_the_box(mesh_and_points):
    m, pts = mesh_and_points
    assert m.ncells == len(pts)
    np.testing.assert_allclose(m.points, pts, rtol=0, atol=0)
    assert (m.volume > 0).all()
    assert abs(m.volume.sum() - 1.0) < 1e-9
    assert (m.face_area > 0).all()


def test_cells_are_closed_and_faces_give_the_volume(mesh_and_points):
    m, _ = mesh_and_points
    for c in range(m.ncells):
        faces = m.cell_faces[m.cell_face_offset[c]:m.cell_face_offset[c + 1]]
        flux = np.zeros(3)
        vol = 0.0
        for f in faces:
            n = _outward(m, c, f)
            flux += n * m.face_area[f]
            vol += np.dot(n, m.face_cm[f]) * m.face_area[f] / 3.0
            assert c in m.face_cells[f]
        assert np.linalg.norm(flux) < 1e-9 * m.face_area[faces].sum()
        assert abs(vol - m.volume[c]) < 1e-9 * max(m.volume[c], 1e-12) + 1e-14
        # the generator lies inside its cell
        for f in faces:
            assert np.dot(m.points[c] - m.face_cm[f], _outward(m, c, f)) < 0


def test_interior_faces_bisect_their_generators(mesh_and_points):
    m, _ = mesh_and_points
    interior = 0
    for f in range(m.nfaces):
        a, b = m.face_cells[f]
        if a >= m.ncells or b >= m.ncells:   # a box face: the other side is a ghost
            continue
        interior += 1
        pa, pb = m.points[a], m.points[b]
        d = pb - pa
        # the centroid is on the bisector plane, whose normal is the generators' separation
        assert abs(np.dot(m.face_cm[f] - 0.5 * (pa + pb), d)) < 1e-9 * np.dot(d, d)
        n = m.face_normal[f] / np.linalg.norm(m.face_normal[f])
        assert abs(abs(np.dot(n, d / np.linalg.norm(d))) - 1.0) < 1e-9
    assert interior > 0


def test_face_polygons_match_their_areas(mesh_and_points):
    m, _ = mesh_and_points
    for f in range(0, m.nfaces, 7):
        vs = m.vertices[m.face_vertices[m.face_vertex_offset[f]:m.face_vertex_offset[f + 1]]]
        assert len(vs) >= 3
        area = 0.5 * np.linalg.norm(sum(np.cross(vs[i], vs[(i + 1) % len(vs)]) for i in range(len(vs))))
        assert abs(area - m.face_area[f]) < 1e-9 * max(m.face_area[f], 1e-12) + 1e-14


def test_build_is_deterministic(mesh_and_points):
    m, pts = mesh_and_points
    m2 = build_voronoi(pts)
    for k in ("volume", "cell_face_offset", "cell_faces", "face_cells", "face_normal", "face_cm", "face_area",
              "face_vertex_offset", "face_vertices", "vertices"):
        np.testing.assert_array_equal(getattr(m, k), getattr(m2, k), err_msg=k)
