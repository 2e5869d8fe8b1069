"""Shared by the statistical tests: run a solver over seeds and judge two
batches with storm_b200.batchstats (per-cell Welch z of the material
temperature, the step's deposit and the two radiation energies after the last
step; Bonferroni bound on the largest |z|, binomial allowance above 3 sigma,
Bonferroni bound on the cell-summed totals)."""
import json

import numpy as np

from storm_b200 import batchstats
from storm_b200.units import UNITS


def run_batch(make, problem_fn, seeds, steps, on_step=None):
    """(K, 1, 4, ncells) quantities after the last of `steps` steps, one row per
    seed.  `on_step(model, stats)` runs after every step (extra checks)."""
    runs = []
    for s in seeds:
        p = problem_fn(s)
        m = make(p)
        vol = p.volumes()
        prev = m.cells()
        for _ in range(steps):
            st = m.step()
            if on_step is not None:
                on_step(m, st)
            cur = m.cells()
            last = batchstats.step_quantities(prev, cur, vol, UNITS["arad"], UNITS["clight"], p.dt)
            prev = cur
        runs.append(last[None])
        m.close()
    return np.array(runs)


def assert_agree(a, b, label=""):
    res = batchstats.compare(a, b)
    summary = {"label": label, "all": res["all"], "totals": res["totals"]}
    print(json.dumps(summary))
    assert res["all"]["tests"] > 0, summary
    assert res["passed"], summary
    return res
