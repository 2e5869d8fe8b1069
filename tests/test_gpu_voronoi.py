"""Gray IMC on a convex-polyhedral (Voronoi) mesh on the GPU against the
reference built on the same mesh (the grid stand-in's polyhedral mode).

* Recorded reference segments (tests/golden/replay_voronoi.npz, with its mesh)
  replay with the same event, destination cell or ghost, and draw count, and
  positions, directions, weights and tallies to the replay tolerances: the face
  search over the cells' inward normals and face centroids, Random Walk
  distances and shrink loop, and the manager's nudges toward mesh points.
* Cell emission puts every packet inside its polyhedron, uniformly (per-cell
  mean position at the cell's centroid within the sampling error).
* Whole steps conserve energy and agree with the reference's serial path
  within the seed-to-seed scatter.
* DDMC-style leakage on polyhedral cells: recorded reference segments
  (tests/golden/replay_voronoi_ddmc.npz) replay, and whole steps agree with
  the reference and between the two forms.
"""
import numpy as np
import pytest

from conftest import golden
from storm_b200 import problems
from storm_b200.engine import Engine
from storm_b200.mesh import PolyMesh, build_voronoi

from test_gpu_parity import _check_replay
from polysample import two_pass_point as _two_pass_point

pytestmark = pytest.mark.gpu

MESH_FIELDS = ("box", "points", "volume", "cell_face_offset", "cell_faces", "face_cells", "face_normal", "face_cm",
               "face_area", "face_vertex_offset", "face_vertices", "vertices")


def _fixture_mesh(g):
    return PolyMesh(*[g["mesh_" + k] for k in MESH_FIELDS])


def test_voronoi_replay_matches_reference(oracle_lib):
    g = golden("replay_voronoi.npz")
    mesh = _fixture_mesh(g)
    p = problems.voronoi_cube(ncells=300, packets_per_step=3e4, seed=21, kappa_median=30.0, mesh=mesh)
    e = Engine(p)
    b = oracle_lib.ReplayBatch(g["before"], g["cell"], g["tape_offset"], g["tape_length"], g["tape"])
    e.set_cell_physics(g["sigma_a"], np.zeros(e.n), g["fleck"])
    e.replay(b)
    same, n = _check_replay(b, g, p.ncells)
    np.testing.assert_array_equal(b["used_random_walk"], g["used_rw"])
    assert (g["next"] >= p.ncells).sum() > 100 and (g["used_rw"] == 1).sum() > 50
    e.close()


def _centroids(mesh):
    """Volume centroid of each cell from the fan tetrahedra about its mesh point."""
    n = mesh.ncells
    cen = np.zeros((n, 3))
    for c in range(n):
        m = mesh.points[c]
        acc, vol = np.zeros(3), 0.0
        for f in mesh.cell_faces[mesh.cell_face_offset[c]:mesh.cell_face_offset[c + 1]]:
            vs = mesh.vertices[mesh.face_vertices[mesh.face_vertex_offset[f]:mesh.face_vertex_offset[f + 1]]]
            for t in range(1, len(vs) - 1):
                a, b, d = vs[0], vs[t], vs[t + 1]
                v = abs(np.dot(a - m, np.cross(b - m, d - m)))
                acc += v * (a + b + d + m) / 4.0
                vol += v
        cen[c] = acc / vol
    return cen


def test_voronoi_cell_emission_inside_and_uniform():
    mesh = build_voronoi(np.random.default_rng(4).random((60, 3)) * 0.98 + 0.01)
    p = problems.voronoi_cube(ncells=60, packets_per_step=6e4, seed=4, mesh=mesh)
    e = Engine(p)
    e.phase("begin", p.dt)
    e.phase("prestep", p.dt)
    e.phase("emit", p.dt)
    b = e.bank()
    cell = b.cell.astype(np.int64)
    pos = np.stack([b.x, b.y, b.z], 1)
    # inside every face plane of its cell (to rounding)
    for c in range(mesh.ncells):
        sel = cell == c
        for f in mesh.cell_faces[mesh.cell_face_offset[c]:mesh.cell_face_offset[c + 1]]:
            nrm, q = mesh.face_normal[f], mesh.face_cm[f]
            side = np.sign(np.dot(mesh.points[c] - q, nrm))
            assert (side * ((pos[sel] - q) @ nrm) >= -1e-12).all(), (c, f)
    cen = _centroids(mesh)
    for c in range(mesh.ncells):
        pc = pos[cell == c]
        se = pc.std(0) / np.sqrt(len(pc))
        assert (np.abs(pc.mean(0) - cen[c]) < 5 * se + 1e-12).all(), c
    e.close()


def test_voronoi_cell_emission_matches_two_pass_sampler(oracle_lib):
    """The device looks the picked tetrahedron up in the mesh's table of running
    volume sums; on the same Philox draws (stream TAG_CELL_EMIT, draws 0-3) the
    positions equal the two-pass sum's bit for bit."""
    mesh = build_voronoi(np.random.default_rng(7).random((40, 3)) * 0.98 + 0.01)
    p = problems.voronoi_cube(ncells=40, packets_per_step=4e3, seed=11, mesh=mesh)
    e = Engine(p)
    e.phase("begin", p.dt)
    e.phase("prestep", p.dt)
    e.phase("emit", p.dt)
    b, st = e.bank(), e.stats()
    e.close()
    n0, ne = int(st["census_in"]), int(st["emitted_cells"])
    assert n0 == 0 and ne > 1000
    box = mesh.box
    checked = 0
    for j in range(ne):
        q = n0 + j
        pid = int(b.id[q])
        u = [oracle_lib.uniform(p.seed, 2, 0, pid, d) for d in range(4)]
        x, y, z = _two_pass_point(mesh, int(b.cell[q]), u)
        if not (box[0] <= x <= box[3] and box[1] <= y <= box[4] and box[2] <= z <= box[5]):
            continue   # moved inside by the outside-box repair
        assert (b.x[q], b.y[q], b.z[q]) == (x, y, z), (j, pid)
        checked += 1
    assert checked > 0.99 * ne


def _balance(st):
    src = st["energy_census_in"] + st["energy_emitted"]
    sink = st["energy_deposited"] + st["energy_escaped"] + st["energy_census_pre_comb"]
    return abs(src - sink) / max(src, 1e-300)


def test_voronoi_steps_conserve_and_agree_with_reference(ref_lib):
    mesh = build_voronoi(np.random.default_rng(8).random((400, 3)) * 0.98 + 0.01)

    from batchcheck import assert_agree, run_batch

    def prob(s):
        p = problems.voronoi_cube(ncells=400, packets_per_step=2e4, seed=8, mesh=mesh)
        p.seed = s
        return p

    def check(m, st):
        if isinstance(m, Engine):
            assert _balance(st) < 1e-10
    assert_agree(run_batch(Engine, prob, range(20, 36), 4, check),
                 run_batch(ref_lib.Reference, prob, range(60, 76), 4), "Voronoi 400 cells: engine vs reference")


def test_voronoi_fp32_tracking_agrees_with_fp64():
    """The FP32-tracking form on polyhedral cells (offsets from the mesh point,
    face planes n.q + h = 0 in FP32): energy conserved per step, the census
    inside its cells, temperatures within the seed-to-seed scatter of the FP64
    form."""
    from storm_b200 import _abi as A
    mesh = build_voronoi(np.random.default_rng(9).random((400, 3)) * 0.98 + 0.01)

    from batchcheck import assert_agree, run_batch

    def prob(precision):
        def make(s):
            p = problems.voronoi_cube(ncells=400, packets_per_step=2e4, seed=9, mesh=mesh, precision=precision)
            p.seed = s
            return p
        return make
    steps_seen = []

    def check(e, st):
        assert _balance(st) < 1e-10
        steps_seen.append(1)
        if len(steps_seen) % 4:
            return
        c = e.census()   # after each run's last step: a sample of the census lies inside its cells
        pos = np.stack([c.x, c.y, c.z], 1)
        cell = c.cell.astype(np.int64)
        for q in np.random.default_rng(len(steps_seen)).choice(len(cell), 300, replace=False):
            k = cell[q]
            for f in mesh.cell_faces[mesh.cell_face_offset[k]:mesh.cell_face_offset[k + 1]]:
                nrm, fc = mesh.face_normal[f], mesh.face_cm[f]
                side = np.sign(np.dot(mesh.points[k] - fc, nrm))
                assert side * np.dot(pos[q] - fc, nrm) >= -1e-7, (k, f)
    assert_agree(run_batch(Engine, prob(A.PRECISION_FP32_TRACK), range(30, 46), 4, check),
                 run_batch(Engine, prob(A.PRECISION_FP64), range(70, 86), 4, check), "Voronoi 400 cells: FP32 vs FP64")


def _face_source_problem(mesh, seed, precision=None):
    from storm_b200 import _abi as A
    from storm_b200.units import UNITS
    p = problems.voronoi_cube(ncells=mesh.ncells, packets_per_step=2e4, seed=11, mesh=mesh)
    p.seed = seed
    p.faces[0] = problems.BoxFace(A.FACE_ESCAPE, 0.5 * UNITS["kev_kelvin"], 20)   # x-low: escape and a 0.5 keV source
    if precision is not None:
        p.precision = precision
    return p


def _x_low_faces(mesh):
    """The mesh's faces on the x-low box plane."""
    return [f for c in range(mesh.ncells)
            for f in mesh.cell_faces[mesh.cell_face_offset[c]:mesh.cell_face_offset[c + 1]]
            if mesh.face_cells[f, 1] >= mesh.ncells and abs(mesh.face_cm[f, 0] - mesh.box[0]) < 1e-12]


def test_voronoi_face_source_matches_reference(ref_lib):
    """A Planck source on the x-low box face of a Voronoi mesh (the boundary
    plug-in over the mesh's polygonal box faces, RandomPointOnFace's fan
    triangles): 20 packets per x-low face, every packet on the face plane moving
    into the box, each with the face's share sigma T^4 A dt / N; then whole
    steps against the reference's serial path on the same mesh under the batch
    gate, and the FP32 form against the FP64 form."""
    from batchcheck import assert_agree, run_batch
    from storm_b200 import _abi as A
    from storm_b200.units import UNITS
    mesh = build_voronoi(np.random.default_rng(11).random((300, 3)) * 0.98 + 0.01)
    faces = _x_low_faces(mesh)
    nf = len(faces)
    assert nf > 5
    p = _face_source_problem(mesh, 5)
    e = Engine(p)
    for ph in ("begin", "prestep", "emit"):
        e.phase(ph)
    st = e.stats()
    assert st["emitted_faces"] == 20 * nf
    b = e.bank()
    face = slice(b.n - 20 * nf, b.n)
    assert np.abs(b.x[face] - mesh.box[0]).max() < 1e-12 and (b.vx[face] > 0).all()
    T = p.faces[0].source_temperature
    total = b.weight[face].sum()
    area = sum(mesh.face_area[f] for f in faces)
    assert abs(total - UNITS["sigma_sb"] * T ** 4 * area * p.dt) < 1e-10 * total
    e.close()
    prob = lambda s: _face_source_problem(mesh, s)   # noqa: E731
    assert_agree(run_batch(Engine, prob, range(20, 36), 4), run_batch(ref_lib.Reference, prob, range(60, 76), 4),
                 "Voronoi 300 cells with an x-low face source: engine vs reference")
    prob32 = lambda s: _face_source_problem(mesh, s, A.PRECISION_FP32_TRACK)   # noqa: E731
    assert_agree(run_batch(Engine, prob32, range(120, 136), 4), run_batch(Engine, prob, range(160, 176), 4),
                 "Voronoi 300 cells with an x-low face source: FP32 vs FP64")


def _ddmc_problem(mesh, seed, precision=None):
    from storm_b200 import _abi as A
    p = problems.voronoi_ddmc(ncells=mesh.ncells, packets_per_step=2e4, mesh=mesh,
                              precision=A.PRECISION_FP64 if precision is None else precision)
    p.seed = seed
    return p


def test_voronoi_ddmc_replay_matches_reference(oracle_lib):
    """DDMC on polyhedral cells (radiation/RadiationIMC.hpp:1282-1612):
    recorded reference segments on a 300-cell Voronoi mesh whose scattering
    half is DDMC eligible (tests/golden/replay_voronoi_ddmc.npz) replay with
    the same event, destination cell and draw count, the same DDMC choice, and
    positions (the leak face's centroid), directions (the cosine law about the
    face normal turned toward the neighbour), weights and tallies to the
    replay tolerances."""
    g = golden("replay_voronoi_ddmc.npz")
    mesh = _fixture_mesh(g)
    p = problems.voronoi_ddmc(mesh=mesh)
    e = Engine(p)
    e.set_cell_state(g["T_start"], None, None)
    e.phase("prestep", p.dt)
    b = oracle_lib.ReplayBatch(g["before"], g["cell"], g["tape_offset"], g["tape_length"], g["tape"])
    e.replay(b)
    _check_replay(b, g, p.ncells, time_rel=1e-13)
    np.testing.assert_array_equal(b["used_random_walk"], g["used_rw"])
    ddmc = g["used_rw"] == 2
    leaks = ddmc & (g["status"] == 1)
    assert leaks.sum() > 500 and (ddmc & (g["status"] == 2)).sum() > 200
    assert len(set(g["next"][leaks].tolist())) > 50   # leaks into many different neighbours
    e.close()


def test_voronoi_ddmc_steps_agree_with_reference(ref_lib):
    """Whole steps with DDMC on a Voronoi mesh: energy conserved per step in
    both forms; the engine against the reference's serial path and the FP32
    form against the FP64 form under the batch gate."""
    from storm_b200 import _abi as A
    from batchcheck import assert_agree, run_batch
    mesh = build_voronoi(np.random.default_rng(12).random((300, 3)) * 0.98 + 0.01)

    def check(m, st):
        if isinstance(m, Engine):
            assert _balance(st) < 1e-10
    fp64 = run_batch(Engine, lambda s: _ddmc_problem(mesh, s), range(20, 36), 4, check)
    assert_agree(fp64, run_batch(ref_lib.Reference, lambda s: _ddmc_problem(mesh, s), range(60, 76), 4),
                 "Voronoi DDMC 300 cells: engine vs reference")
    assert_agree(run_batch(Engine, lambda s: _ddmc_problem(mesh, s, A.PRECISION_FP32_TRACK), range(40, 56), 4, check),
                 fp64, "Voronoi DDMC 300 cells: FP32 vs FP64")
