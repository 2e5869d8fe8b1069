"""Run the reference's full-run benchmarks through the reference build
(oracle/_ref/libstormref.so: STORM's serial manager and RadiationIMC compiled
from the reference sources) and pack their final profiles into
reference_runs.npz.  Each problem runs in a fresh process, because
CombPopulationControl and the boundary sources keep function-static random
engines.  Run where the reference sources were compiled:

    make -C oracle all REF=<reference source tree> && python tests/golden/make_reference_runs.py

Arrays, per problem name (marshak_wave_1..4 at the examples' defaults: 256
cells (512 for problem 4), 15 packets per cell, 100 per bath face, comb
(15, 6); densmore2012 at 512 cells, 16 per cell, 100 per face, comb (200, 5); densmore2012_small at 128 cells, 8 per cell,
comb (50, 5)):
  <name>_x, <name>_t_gas, <name>_t_rad   final profile sorted by x [cm, K, K]
  <name>_l1                              the example's L1 against its published curve
  <name>_wall                            seconds the run took on one core
"""
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

PROBLEMS = ["marshak_wave_1", "marshak_wave_2", "marshak_wave_3", "marshak_wave_4", "densmore2012",
            "densmore2012_small"]
# densmore2012_small: the Densmore slab at 128 cells, 8 packets per cell, comb Nmin 50 (the example's
# default size takes the reference's serial path hours on one core)
DENSMORE_SMALL = dict(nx=128, new_photons_per_cell=8, boundary_per_face=100, comb_nmin=50)


def run_one(name):
    from oracle import ref
    from storm_b200 import benchmarks as B
    curves = np.load(os.path.join(HERE, "reference_curves.npz"))
    t0 = time.time()
    if name.startswith("densmore2012"):
        res = B.run_densmore2012(ref.Reference, **(DENSMORE_SMALL if name.endswith("_small") else {}))
        l1 = B.densmore_l1(res["x"], res["t_gas"], curves["densmore2012"])
    else:
        k = int(name[-1])
        res = B.run_marshak_wave(ref.Reference, k)
        l1 = B.marshak_l1(res["x"], res["t_gas"], curves[name])
    return name, res, l1, time.time() - t0


def main(names):
    ctx = mp.get_context("spawn")
    path = os.path.join(HERE, "reference_runs.npz")
    new = {}
    with ctx.Pool(len(names), maxtasksperchild=1) as pool:
        for name, res, l1, wall in pool.imap_unordered(run_one, names):
            print(f"{name}: L1 {l1:.4e}, {res['steps']} steps, {wall:.0f} s", flush=True)
            for k in ("x", "t_gas", "t_rad"):
                new[f"{name}_{k}"] = res[k]
            new[f"{name}_l1"] = np.float64(l1)
            new[f"{name}_wall"] = np.float64(wall)
    # problems not rerun keep their earlier results (read now: other runs may have written meanwhile)
    out = dict(np.load(path)) if os.path.exists(path) else {}
    for name in names:
        for k in [k for k in out if k.startswith(name + "_")]:
            del out[k]
    out.update(new)
    np.savez_compressed(path, **out)


if __name__ == "__main__":
    main(sys.argv[1:] or PROBLEMS)
