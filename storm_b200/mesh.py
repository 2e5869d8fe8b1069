"""Convex-polyhedral meshes: a bounded Voronoi tessellation built by the
engine's library (storm_mesh_voronoi), held as numpy arrays in the C ABI's
StormPolyMesh layout.  The reference takes its Voronoi grids from MadVoro;
this is the engine's own builder."""
import ctypes as C

import numpy as np

from . import _abi as A


class PolyMesh:
    """A mesh in the StormPolyMesh layout.  `build_voronoi` makes one from
    generator points; the arrays are copied out of the library, so the object
    owns them and `desc()` points a StormPolyMesh at them."""

    def __init__(self, box, points, volume, cell_face_offset, cell_faces, face_cells, face_normal, face_cm,
                 face_area, face_vertex_offset, face_vertices, vertices):
        self.box = np.asarray(box, np.float64)
        self.points = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
        self.volume = np.ascontiguousarray(volume, np.float64)
        self.cell_face_offset = np.ascontiguousarray(cell_face_offset, np.uint32)
        self.cell_faces = np.ascontiguousarray(cell_faces, np.uint32)
        self.face_cells = np.ascontiguousarray(face_cells, np.uint32).reshape(-1, 2)
        self.face_normal = np.ascontiguousarray(face_normal, np.float64).reshape(-1, 3)
        self.face_cm = np.ascontiguousarray(face_cm, np.float64).reshape(-1, 3)
        self.face_area = np.ascontiguousarray(face_area, np.float64)
        self.face_vertex_offset = np.ascontiguousarray(face_vertex_offset, np.uint32)
        self.face_vertices = np.ascontiguousarray(face_vertices, np.uint32)
        self.vertices = np.ascontiguousarray(vertices, np.float64).reshape(-1, 3)
        self._desc = None

    @property
    def ncells(self):
        return len(self.volume)

    @property
    def nfaces(self):
        return len(self.face_area)

    def desc(self):
        m = A.StormPolyMesh()
        m.ncells, m.nfaces, m.nvertices = self.ncells, self.nfaces, len(self.vertices)
        for k in range(6):
            m.box[k] = self.box[k]
        m.points, m.volume = A.ptr(self.points), A.ptr(self.volume)
        m.cell_face_offset = A.ptr(self.cell_face_offset, C.c_uint32)
        m.cell_faces = A.ptr(self.cell_faces, C.c_uint32)
        m.face_cells = A.ptr(self.face_cells, C.c_uint32)
        m.face_normal, m.face_cm, m.face_area = A.ptr(self.face_normal), A.ptr(self.face_cm), A.ptr(self.face_area)
        m.face_vertex_offset = A.ptr(self.face_vertex_offset, C.c_uint32)
        m.face_vertices = A.ptr(self.face_vertices, C.c_uint32)
        m.vertices = A.ptr(self.vertices)
        self._desc = m
        return m

    def surface(self):
        """Per cell, the sum of its face areas in face order."""
        s = np.zeros(self.ncells)
        for c in range(self.ncells):
            a, b = self.cell_face_offset[c], self.cell_face_offset[c + 1]
            for f in self.cell_faces[a:b]:
                s[c] += self.face_area[f]
        return s


def build_voronoi(points, box=(0.0, 0.0, 0.0, 1.0, 1.0, 1.0)):
    """The bounded Voronoi tessellation of `points` ((n, 3), strictly inside the box)."""
    from .engine import lib
    L = lib()
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    b = (C.c_double * 6)(*box)
    out = C.POINTER(A.StormPolyMesh)()
    rc = L.storm_mesh_voronoi(A.ptr(pts), len(pts), b, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"storm_mesh_voronoi failed ({rc})")
    m = out.contents
    n, F, V = m.ncells, m.nfaces, m.nvertices

    def arr(p, k, dtype):
        return np.ctypeslib.as_array(p, (k,)).astype(dtype).copy()
    cfo = arr(m.cell_face_offset, n + 1, np.uint32)
    fvo = arr(m.face_vertex_offset, F + 1, np.uint32)
    mesh = PolyMesh(box, arr(m.points, 3 * n, np.float64), arr(m.volume, n, np.float64), cfo,
                    arr(m.cell_faces, int(cfo[-1]), np.uint32), arr(m.face_cells, 2 * F, np.uint32),
                    arr(m.face_normal, 3 * F, np.float64), arr(m.face_cm, 3 * F, np.float64),
                    arr(m.face_area, F, np.float64), fvo, arr(m.face_vertices, int(fvo[-1]), np.uint32),
                    arr(m.vertices, 3 * V, np.float64))
    L.storm_mesh_free(out)
    return mesh
