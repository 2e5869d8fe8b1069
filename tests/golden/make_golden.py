"""Generate the golden fixtures in this directory from the reference build
(oracle/_ref/libstormref.so: STORM's own serial path compiled from the reference
sources against oracle/shims).  Run in a container where the reference sources
are present:

    make -C oracle all REF=<reference source tree> && python tests/golden/make_golden.py

Fixtures (numpy .npz):
  replay_slab.npz     recorded RadiationIMC::step calls on the gray slab (boundary
                      reflect / escape, face crossings, collisions, census, cutoff)
  replay_cube_rw.npz  recorded calls on an 8^3 step-opacity cube with Random Walk
  rw_samples.npz      RandomWalk::sampleLeakTime / sampleRadius at seeded points
  samplers.npz        RandomInCellPositionSampler / isotropicVelocity /
                      RandomPointOnFace outputs with the draws each consumed
  allocation_slab.npz photon counts per cell (getLastSourcePhotonsPerCell) and the
                      cell temperatures they were allocated from, several steps
  replay_mg.npz       recorded calls on a 6^3 multigroup cube (64 groups, PGRW)
                      with frequencies and the step's starting temperatures
  replay_mg_thin.npz  the same, optically thinner, opacity continuous in frequency
  replay_ddmc.npz     recorded calls on an 8^3 step cube with DDMC leakage (withDDMC)
                      and the step's starting temperatures
  replay_ddmc_rw.npz  the same with Random Walk on (particle depth 20): Random Walk
                      jumps where deep enough, DDMC steps between depths 5 and 20
  replay_ddmc_mg.npz  a 64-group cube with DDMC in its multigroup PGRW form
  replay_voronoi.npz  recorded calls on a 300-cell Voronoi mesh (Random Walk on), with
                      the mesh arrays (mesh_*)
  replay_voronoi_ddmc.npz  recorded calls on a 300-cell Voronoi mesh with DDMC leakage
                      in its scattering half (problems.voronoi_ddmc), with the mesh
                      arrays and the step's starting temperatures
  replay_hydro.npz    recorded calls on an 8^3 step cube (Random Walk, elastic
                      scattering in the thin half) whose cells move at up to 5 % of c
                      (withHydro), with the velocities and each segment's momentum deposit
  replay_hydro_mg.npz the same for a 64-group cube with PGRW

    python tests/golden/make_golden.py ddmc     # only the DDMC fixtures
    python tests/golden/make_golden.py voronoi  # only the Voronoi fixtures
    python tests/golden/make_golden.py hydro    # only the moving-material fixtures
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from storm_b200 import problems  # noqa: E402


def record(problem, warm_steps, max_records, take, mg=False):
    r = ref.Reference(problem)
    for _ in range(warm_steps):
        r.step()
    c = r.cells()     # tables of the last step; the recorded step recomputes them
    T_start = c["temperature"]
    vel_start = r.motion()[0] if problem.with_hydro else None
    r.record_begin(max_records)
    r.step()
    r.record_end()
    rec = r.records()
    c = r.cells()
    n = len(rec["cell"])
    # keep a deterministic, representative subset: every k-th record plus all
    # boundary interactions and Random Walk jumps
    idx = np.arange(n)
    special = (rec["status"] == 1) & (rec["next"] >= problem.ncells)
    special |= rec["used_rw"] != 0   # Random Walk jumps and DDMC steps
    special |= rec["status"] == 3
    if mg:   # every frequency change (effective scatters, PGRW upscatters)
        special |= rec["freq_before"] != rec["freq_after"]
    sub = idx[(idx % max(1, n // take) == 0) | special]
    if len(sub) > 3 * take:
        sub = sub[np.linspace(0, len(sub) - 1, 3 * take).astype(int)]
    tape_off = rec["tape_offset"][sub]
    tape_len = rec["tape_length"][sub]
    tape = np.concatenate([rec["tape"][o:o + l] for o, l in zip(tape_off, tape_len)]) if len(sub) else np.zeros(0)
    new_off = np.concatenate([[0], np.cumsum(tape_len)[:-1]]).astype(np.uint64)
    # chained successor (the same particle's next record) for the manager check
    nxt_before = np.full((len(sub), 6), np.nan)
    nxt_cell = np.full(len(sub), -1, np.int64)
    for q, k in enumerate(sub):
        if k + 1 < n and rec["id"][k + 1] == rec["id"][k]:
            nxt_before[q] = rec["before"][k + 1][:6]
            nxt_cell[q] = rec["cell"][k + 1]
    out = dict(before=rec["before"][sub], after=rec["after"][sub], status=rec["status"][sub],
               next=rec["next"][sub].astype(np.int64), tallies=rec["tallies"][sub], cell=rec["cell"][sub],
               used_rw=rec["used_rw"][sub], tape=tape, tape_offset=new_off, tape_length=tape_len,
               next_before=nxt_before, next_cell=nxt_cell, sigma_a=c["sigma_a"], fleck=c["fleck"])
    if mg:   # frequencies, and the temperatures the recorded step built its tables from
        out.update(freq_before=rec["freq_before"][sub], freq_after=rec["freq_after"][sub], T_start=T_start)
    if problem.with_ddmc:
        out.update(T_start=T_start)
    if problem.with_hydro:   # the cells' velocities at the recorded step, and each segment's momentum deposit
        out.update(T_start=T_start, vel_start=vel_start, momentum=rec["momentum"][sub])
    return out


def hydro_velocity(p, beta=0.05):
    """A smooth velocity field of the cells, |v| up to about beta c."""
    from storm_b200.units import UNITS
    xc, yc, zc = p.cell_centers()
    v = np.stack([np.sin(2 * np.pi * yc), np.cos(2 * np.pi * xc), 0.5 * np.sin(2 * np.pi * zc)], 1)
    return v * (beta * UNITS["clight"])


def hydro_problems():
    """The moving-material fixtures' problems (withHydro, cells moving at up to 5 % of c)."""
    gray = problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20, seed=31)
    gray.sigma_s = np.where(gray.cell_centers()[0] < 0.5, 2.0, 0.0)   # elastic scatters too
    gray.with_hydro = True
    gray.cell_velocity = hydro_velocity(gray)
    mg = problems.mg_cube(n=6, groups=64, new_photons_per_cell=3, comb_nmin=3, seed=32)
    mg.with_hydro = True
    mg.cell_velocity = hydro_velocity(mg)
    return {"replay_hydro.npz": gray, "replay_hydro_mg.npz": mg}


def make_hydro():
    for name, p in hydro_problems().items():
        np.savez_compressed(os.path.join(HERE, name), **record(p, 1, 400000, 1500, mg=p.groups >= 2))


def make_ddmc():
    gray = problems.ddmc_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20, seed=11)
    np.savez_compressed(os.path.join(HERE, "replay_ddmc.npz"), **record(gray, 1, 400000, 1500))
    mixed = problems.ddmc_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20, seed=12,
                               with_random_walk=True, rw_min_particle_optical_depth=20.0)
    np.savez_compressed(os.path.join(HERE, "replay_ddmc_rw.npz"), **record(mixed, 1, 400000, 1500))
    mg = problems.mg_cube(n=6, groups=64, kappa0=1e-4, new_photons_per_cell=3, comb_nmin=3, seed=13, dt=1e-10,
                          with_random_walk=False)
    mg.sigma_s = np.full(mg.ncells, 1000.0)
    mg.with_ddmc = True
    mg.ddmc_use_multigroup_pgrw = True
    np.savez_compressed(os.path.join(HERE, "replay_ddmc_mg.npz"), **record(mg, 1, 400000, 1500, mg=True))


def main():
    slab = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50)
    np.savez_compressed(os.path.join(HERE, "replay_slab.npz"), **record(slab, 2, 400000, 1500))

    cube = problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20)
    np.savez_compressed(os.path.join(HERE, "replay_cube_rw.npz"), **record(cube, 1, 400000, 1500))

    # multigroup: 64 groups, PGRW, group-constant kappa0 nu^-3 (1 - e^{-nu/T}) (replay_mg.npz)
    mg = problems.mg_cube(n=6, groups=64, new_photons_per_cell=3, comb_nmin=3, seed=5)
    np.savez_compressed(os.path.join(HERE, "replay_mg.npz"), **record(mg, 1, 400000, 1500, mg=True))
    # optically thinner, opacity continuous in frequency: collisions, effective scatters, face crossings
    mgt = problems.mg_cube(n=6, groups=64, kappa0=1.0, new_photons_per_cell=3, comb_nmin=3, seed=6,
                           group_constant=False)
    np.savez_compressed(os.path.join(HERE, "replay_mg_thin.npz"), **record(mgt, 1, 400000, 1500, mg=True))

    rng = np.random.default_rng(7)
    xi_leak = np.concatenate([rng.random(3000), [1e-300, 1e-12, 0.5, 1 - 1e-12, np.nextafter(1, 0)]])
    tau = np.concatenate([10 ** rng.uniform(-10, 2.5, 3000), [1e-9, 1e-8, 64.0, 100.0, 0.01]])
    xi_rad = np.concatenate([rng.random(3000), [0.0, 1.0, 0.5, 1e-9, 1 - 1e-9]])
    leak, rad = ref.rw_sample(xi_leak, tau, xi_rad)
    t_grid = 10 ** np.linspace(-9, 2, 400)
    x_grid = rng.random(400)
    surv, cdf = ref.rw_functions(t_grid, x_grid)
    np.savez_compressed(os.path.join(HERE, "rw_samples.npz"), xi_leak=xi_leak, tau=tau, xi_rad=xi_rad, leak=leak,
                        radius=rad, t_grid=t_grid, x_grid=x_grid, survival=surv, cdf=cdf)

    small = problems.step_cube(n=4)
    rs = ref.Reference(small)
    cells = rng.integers(0, small.ncells, 500).astype(np.uint32)
    pos, ptape, nd = rs.sample_in_cell(cells, 12345)
    vel, vtape = ref.isotropic(500, 99)
    nxf = 5 * 4 * 4
    faces = rng.integers(0, 3 * nxf, 300).astype(np.uint64)
    fpos, ftape = rs.point_on_face(faces)
    np.savez_compressed(os.path.join(HERE, "samplers.npz"), cells=cells, cell_pos=pos, cell_tape=ptape,
                        cell_draws=nd, vel=vel, vel_tape=vtape, faces=faces, face_pos=fpos, face_tape=ftape,
                        x_edges=small.x_edges, y_edges=small.y_edges, z_edges=small.z_edges)

    slab2 = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50)
    r2 = ref.Reference(slab2)
    T_before, counts, eint_before, sig, fl = [], [], [], [], []
    for _ in range(4):
        c = r2.cells()
        T_before.append(c["temperature"])
        eint_before.append(c["internal_energy"])
        r2.step()
        counts.append(r2.emission_counts())
        c = r2.cells()
        sig.append(c["sigma_a"])
        fl.append(c["fleck"])
    np.savez_compressed(os.path.join(HERE, "allocation_slab.npz"), temperature=np.array(T_before),
                        internal_energy=np.array(eint_before), photons=np.array(counts), sigma_a=np.array(sig),
                        fleck=np.array(fl))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


MESH_FIELDS = ("box", "points", "volume", "cell_face_offset", "cell_faces", "face_cells", "face_normal", "face_cm",
               "face_area", "face_vertex_offset", "face_vertices", "vertices")


def voronoi_problem(mesh=None):
    """The Voronoi fixture's problem: 300 cells, kappa lognormal about 30 1/cm."""
    return problems.voronoi_cube(ncells=300, packets_per_step=3e4, seed=21, kappa_median=30.0, mesh=mesh)


def make_voronoi():
    p = voronoi_problem()
    out = record(p, 1, 400000, 1500)
    out.update({"mesh_" + k: getattr(p.mesh, k) for k in MESH_FIELDS})
    np.savez_compressed(os.path.join(HERE, "replay_voronoi.npz"), **out)


def make_voronoi_ddmc():
    p = problems.voronoi_ddmc()
    out = record(p, 1, 400000, 1500)
    out.update({"mesh_" + k: getattr(p.mesh, k) for k in MESH_FIELDS})
    np.savez_compressed(os.path.join(HERE, "replay_voronoi_ddmc.npz"), **out)


if __name__ == "__main__":
    if sys.argv[1:] == ["ddmc"]:
        make_ddmc()
    elif sys.argv[1:] == ["voronoi"]:
        make_voronoi()
        make_voronoi_ddmc()
    elif sys.argv[1:] == ["hydro"]:
        make_hydro()
    else:
        main()
        make_ddmc()
        make_voronoi()
        make_voronoi_ddmc()
        make_hydro()
