"""Batch runs of the reference's serial path (oracle/_ref/libstormref.so: STORM's
MonteCarloManagerSerial + RadiationIMC + CombPopulationControl compiled from
the reference sources) over independent seeds, summarised per cell into
reference_batch.npz for the full-run parity tests (tests/test_gpu_fullrun.py).

Each seed runs in a fresh process: CombPopulationControl seeds its
function-static engine from the first census size, and RandomPointOnFace
keeps a function-static std::mt19937(0), which each run moves forward by
FACE_STREAM_SPACING x (run index) points before its first step.  The
harness's boundary takes its own engine's seed from the problem seed.

Run where the reference sources were compiled:

    make -C oracle ref REF=<reference source tree> && python tests/golden/make_reference_batch.py [c1] [c2r] [marshak1]

Workloads (storm_b200.problems):
  c1   the 100x1x1 gray slab at its defaults (about 1e5 source packets and
       1e5 census particles per step, comb Nmin 500 factor 2), 100 steps of
       dt = 1e-11 s, recorded after steps 1, 5, 20, 50, 100; 32 seeds
  c2r  the two-material step-opacity cube with Random Walk, cut from 64^3
       to 16^3 cells at the same per-cell and per-face packet densities
       (3 per cell, 450 per x=0 face, comb Nmin 20 factor 2: about 2.5e5
       source packets per step), 20 steps, recorded after steps 1, 10, 20;
       24 seeds
  marshak1  Marshak wave 1 (examples/marshak_wave) at the example's defaults,
       7,912 steps to 1 ns with the bath updated before each step; 24 seeds
Arrays per workload <w>: batchstats.summary_for_fixture of the runs
(<w>_mean, <w>_var, <w>_n, <w>_nonzero, <w>_total_*), <w>_snapshots,
<w>_seeds and <w>_wall (seconds per run).  For marshak1 instead: the final
gas temperature of every run (marshak1_t_gas, sorted by x), marshak1_x and
the example's L1 of every run against its published curve (marshak1_l1).
"""
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FACE_STREAM_SPACING = 1 << 23


def workload(name, seed):
    from storm_b200 import problems
    if name == "c1":
        return problems.gray_slab(seed=seed)
    if name == "c2r":
        return problems.step_cube(n=16, new_photons_per_cell=3, face_packets=450, comb_nmin=20, comb_factor=2.0,
                                  seed=seed)
    raise ValueError(name)


WORKLOADS = {
    "c1": dict(steps=100, snapshots=(1, 5, 20, 50, 100), seeds=list(range(1000, 1032))),
    "c2r": dict(steps=20, snapshots=(1, 10, 20), seeds=list(range(1000, 1024))),
    "marshak1": dict(seeds=list(range(1000, 1024))),
}


def run_marshak(index, seed):
    from oracle import ref
    from storm_b200 import benchmarks as B

    def make(p):
        m = ref.Reference(p)
        m.advance_face_stream(FACE_STREAM_SPACING * index)
        return m
    curve = np.load(os.path.join(HERE, "reference_curves.npz"))["marshak_wave_1"]
    t0 = time.time()
    res = B.run_marshak_wave(make, 1, seed=seed)
    res["l1"] = B.marshak_l1(res["x"], res["t_gas"], curve)
    return "marshak1", index, res, time.time() - t0


def run_one(job):
    name, index, seed = job
    if name == "marshak1":
        return run_marshak(index, seed)
    from oracle import ref
    from storm_b200 import batchstats
    w = WORKLOADS[name]
    p = workload(name, seed)
    m = ref.Reference(p)
    m.advance_face_stream(FACE_STREAM_SPACING * index)
    t0 = time.time()
    snaps = batchstats.run_snapshots(m, p, w["steps"], w["snapshots"])
    m.close()
    return name, index, snaps, time.time() - t0


def main(names):
    from storm_b200 import batchstats
    path = os.path.join(HERE, "reference_batch.npz")
    jobs = [(n, k, s) for n in names for k, s in enumerate(WORKLOADS[n]["seeds"])]
    runs = {n: [None] * len(WORKLOADS[n]["seeds"]) for n in names}
    walls = {n: [] for n in names}
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count(), maxtasksperchild=1) as pool:
        for name, k, snaps, wall in pool.imap_unordered(run_one, jobs):
            runs[name][k] = snaps
            walls[name].append(wall)
            print(f"{name} seed #{k}: {wall:.0f} s", flush=True)
    out = dict(np.load(path)) if os.path.exists(path) else {}
    for name in names:
        for key in [key for key in out if key.startswith(name + "_")]:
            del out[key]
        if name == "marshak1":
            out["marshak1_x"] = runs[name][0]["x"]
            out["marshak1_t_gas"] = np.array([r["t_gas"] for r in runs[name]])
            out["marshak1_l1"] = np.array([r["l1"] for r in runs[name]])
            out["marshak1_seeds"] = np.array(WORKLOADS[name]["seeds"])
            out["marshak1_wall"] = np.float64(np.mean(walls[name]))
            continue
        summ = batchstats.summary_for_fixture(np.array(runs[name]))
        for key, v in summ.items():
            out[f"{name}_{key}"] = v
        out[f"{name}_snapshots"] = np.array(WORKLOADS[name]["snapshots"])
        out[f"{name}_seeds"] = np.array(WORKLOADS[name]["seeds"])
        out[f"{name}_wall"] = np.float64(np.mean(walls[name]))
    np.savez_compressed(path, **out)


if __name__ == "__main__":
    main(sys.argv[1:] or list(WORKLOADS))
