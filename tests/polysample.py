"""The reference's RandomInCellPositionSampler on a convex-polyhedral cell,
restated for the tests (utils/RandomInCell.hpp:11-67): the fan tetrahedra of the
cell's face polygons about its mesh point, picked by volume with the volumes
summed twice (the total, then the running sum up to the pick), then a point
from three sorted uniforms.  Python floats are IEEE doubles and every step is
one rounded operation, as in the reference's build without contraction."""


def two_pass_point(mesh, c, u):
    """RandomInCellPositionSampler on polyhedral cell c (utils/RandomInCell.hpp:11-67)
    from draws u[0..3], summing the fan tetrahedra's volumes twice as the
    reference does: the total, then the running sum up to the picked one."""
    cx, cy, cz = (float(v) for v in mesh.points[c])
    V = mesh.vertices
    tets = []
    for f in mesh.cell_faces[mesh.cell_face_offset[c]:mesh.cell_face_offset[c + 1]]:
        a, b = int(mesh.face_vertex_offset[f]), int(mesh.face_vertex_offset[f + 1])
        for t in range(a + 1, b - 1):
            tets.append((int(mesh.face_vertices[a]), int(mesh.face_vertices[t]), int(mesh.face_vertices[t + 1])))

    def vol(v0, v1, v2):
        ax, ay, az = V[v0, 0] - cx, V[v0, 1] - cy, V[v0, 2] - cz
        bx, by, bz = V[v1, 0] - cx, V[v1, 1] - cy, V[v1, 2] - cz
        ex, ey, ez = V[v2, 0] - cx, V[v2, 1] - cy, V[v2, 2] - cz
        crx, cry, crz = by * ez - bz * ey, bz * ex - bx * ez, bx * ey - by * ex
        return abs(ax * crx + ay * cry + az * crz)

    total = 0.0
    for tt in tets:
        total += vol(*tt)
    r = u[0] * total
    run, pick = 0.0, tets[-1]
    for tt in tets:
        run += vol(*tt)
        if not run < r:
            pick = tt
            break
    s, t, w = sorted((u[1], u[2], u[3]))
    a0, a1, a2, a3 = s, t - s, w - t, 1 - w
    v0, v1, v2 = (V[k] for k in pick)
    return tuple(a0 * v0[d] + a1 * v1[d] + a2 * v2[d] + a3 * (cx, cy, cz)[d] for d in range(3))
