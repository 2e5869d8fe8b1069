"""Batch statistics for full-run parity of two Monte Carlo IMC solvers.

Two solvers (the engine and the reference's serial path, or two precision
forms of the engine) are each run over K independent seeds.  Per cell and per
recorded step they give a batch mean and a batch variance of the quantities
`postStep` leaves behind (`radiation/RadiationIMC.hpp:1887-2029`): the
material temperature, the energy deposited in the material during the step,
the time-averaged radiation energy density and the radiation energy in census.

Their difference is judged in units of its own batch-estimated standard
error (Welch's t, converted to the normal deviate of equal two-sided tail
probability).  `gate` then asks what a correct solver meets with a known
probability:

* no |z| above the Bonferroni bound norm.isf(alpha / (4 M)) for M tests; this
  holds whatever the correlation between tests;
* at most k_max of the M tests above |z| = 3, k_max being the binomial
  quantile of the nominal 0.27 % at probability alpha / 2 (exact for
  independent tests; correlated cells widen the count's spread, which the
  seed-split control of the same solver measures);
* every cell-summed quantity (a total energy) within the Bonferroni bound of
  its own Welch z, which is where a global bias shows first.
"""
import numpy as np

QUANTITIES = ("temperature", "deposit", "erad_time_avg", "erad_census")


def step_quantities(before, after, volume, arad, clight, dt):
    """The per-cell quantities of one step from the cell arrays before and
    after it (`cells()` of either solver): material temperature, deposited
    energy = E_int(after) - E_int(before) + emitted energy, with the emitted
    energy f V a T^4 sigma_P c dt at the step's start temperature
    (`radiation/RadiationIMC.hpp:2058`), and the two radiation energies."""
    emit = after["fleck"] * volume * arad * before["temperature"] ** 4 * after["sigma_a"] * clight * dt
    deposit = after["internal_energy"] - before["internal_energy"] + emit
    return np.stack([after["temperature"], deposit, after["erad_time_avg"], after["erad_census"]])


def run_snapshots(model, problem, steps, snapshots):
    """Run `steps` steps of `model` (an engine or a reference instance: any
    object with step() and cells()) and return an array (len(snapshots),
    len(QUANTITIES), ncells) of the quantities after each recorded step
    (1-based step numbers)."""
    from .units import UNITS
    vol = problem.volumes()
    want = set(snapshots)
    out = []
    prev = model.cells()
    for s in range(1, steps + 1):
        model.step()
        cur = model.cells()
        if s in want:
            out.append(step_quantities(prev, cur, vol, UNITS["arad"], UNITS["clight"], problem.dt))
        prev = cur
    return np.array(out)


def summarize(runs):
    """Batch summary of runs shaped (K, ...): mean, unbiased variance, count,
    and the fraction of runs with a nonzero value per entry."""
    runs = np.asarray(runs, dtype=np.float64)
    return {"mean": runs.mean(0), "var": runs.var(0, ddof=1), "n": runs.shape[0],
            "nonzero": (runs != 0.0).mean(0)}


def welch_z(a, b, floor=None):
    """Normal-equivalent z of Welch's t for mean(a) - mean(b), per entry, with
    a mask of the entries it is defined on.  a and b are `summarize` results.
    Entries where either side is zero in more than a tenth of its runs are
    masked out: there the batch mean is a handful of rare events and a
    t-statistic means nothing.  So are entries whose standard error is below
    `floor` (broadcast against the entries): there the runs differ only by
    rounding, e.g. a cold cell that no particle reached, whose temperature
    the two solvers round differently."""
    from scipy import stats
    va, vb = a["var"] / a["n"], b["var"] / b["n"]
    se2 = va + vb
    ok = np.isfinite(se2) & (se2 > 0) & (a["nonzero"] >= 0.9) & (b["nonzero"] >= 0.9)
    if floor is not None:
        ok &= se2 > np.square(floor)
    t = np.zeros_like(se2)
    df = np.ones_like(se2)
    t[ok] = (a["mean"] - b["mean"])[ok] / np.sqrt(se2[ok])
    den = va ** 2 / max(a["n"] - 1, 1) + vb ** 2 / max(b["n"] - 1, 1)
    df[ok] = se2[ok] ** 2 / np.maximum(den[ok], 1e-300)
    p = 2.0 * stats.t.sf(np.abs(t), df)
    z = np.sign(t) * stats.norm.isf(np.maximum(p, 1e-300) / 2.0)
    return np.where(ok, z, 0.0), ok


def gate(z, alpha=1e-3, threshold=3.0):
    """The pass/fail gate over the z of M tests (see the module text).
    Returns a dict with the counts, the bounds and `passed`."""
    from scipy import stats
    z = np.asarray(z, dtype=np.float64).ravel()
    m = z.size
    if m == 0:
        return {"tests": 0, "passed": False, "why": "no populated tests"}
    p_nominal = 2.0 * stats.norm.sf(threshold)
    above = int(np.sum(np.abs(z) > threshold))
    k_max = int(stats.binom.isf(alpha / 2.0, m, p_nominal))
    z_bound = float(stats.norm.isf(alpha / (4.0 * m)))
    max_abs = float(np.max(np.abs(z)))
    return {"tests": m, "above_threshold": above, "threshold": threshold, "k_max": k_max,
            "expected_above": m * p_nominal, "max_abs_z": max_abs, "z_bound": z_bound,
            "mean_z": float(z.mean()), "rms_z": float(np.sqrt(np.mean(z ** 2))),
            "frac_within": {str(s): float(np.mean(np.abs(z) <= s)) for s in (1, 2, 3)},
            "passed": bool(above <= k_max and max_abs <= z_bound)}


# statistical errors below this fraction of a quantity's largest cell value
# (per recorded step) are rounding, not sampling
RESOLUTION = 1e-9


def compare(runs_a, ref_b, alpha=1e-3):
    """Full comparison of engine runs (K, S, Q, ncells) against a summary of
    the other solver's runs (or its raw runs): the per-cell gate over every
    populated (step, quantity, cell), one gate per quantity for reading, and
    the Welch z of each cell-summed total."""
    a = summarize(runs_a)
    b = ref_b if isinstance(ref_b, dict) else summarize(ref_b)
    scale = np.maximum(np.abs(a["mean"]), np.abs(b["mean"])).max(axis=-1, keepdims=True)
    z, ok = welch_z(a, b, RESOLUTION * scale)
    out = {"all": gate(z[ok], alpha)}
    for q, name in enumerate(QUANTITIES):
        out[name] = gate(z[:, q][ok[:, q]], alpha)
    totals_a = np.asarray(runs_a).sum(-1)
    if isinstance(ref_b, dict):
        tb = {"mean": ref_b["total_mean"], "var": ref_b["total_var"], "n": ref_b["n"],
              "nonzero": ref_b["total_nonzero"]}
    else:
        tb = summarize(np.asarray(ref_b).sum(-1))
    zt, okt = welch_z(summarize(totals_a), tb)
    from scipy import stats
    bound = float(stats.norm.isf(alpha / (2.0 * max(int(okt.sum()), 1))))
    out["totals"] = {"z": zt.tolist(), "max_abs_z": float(np.max(np.abs(zt[okt]))) if okt.any() else 0.0,
                     "z_bound": bound}
    out["passed"] = bool(out["all"]["passed"] and out["totals"]["max_abs_z"] <= bound)
    return out


def summary_for_fixture(runs):
    """What a committed fixture keeps of a batch of runs (K, S, Q, ncells):
    per-entry mean, variance and nonzero fraction, plus the same for the
    cell-summed totals."""
    s = summarize(runs)
    t = summarize(np.asarray(runs).sum(-1))
    return {"mean": s["mean"], "var": s["var"], "n": np.int64(s["n"]), "nonzero": s["nonzero"],
            "total_mean": t["mean"], "total_var": t["var"], "total_nonzero": t["nonzero"]}
