"""The reference's own full-run benchmarks, driven through the engine, with the
accuracy gates its regression suite applies.

* Marshak waves 1-4 (examples/marshak_wave/MarshakCommon.hpp:265-432): gray
  IMC with a power-law opacity and EOS and a time-dependent bath on x=0, on
  the example's geometric time-step schedule to 1 ns.  The gas temperature is
  compared with the diffusion reference profile by the example's relative L1
  (MarshakCommon.hpp:193-228); the regression suite passes it below 0.10
  (regression_tests/lib/regression_checks.sh:73-97).
* Densmore et al. (2012) Fig. 4 (examples/densmore2012/main.cpp): 30 groups,
  opacity sigma0 / (sqrt(kT) E^3) with a step in sigma0, a 1 keV Planck source
  on x=0, 200 steps of 5 ps.  The gas temperature is compared with the
  digitised Milagro curve by the example's absolute L1 in keV
  (main.cpp:315-353); the gate is 0.10 keV.

`make` is any callable that turns a Problem into an object with
``step(dt)``, ``set_face_temperature(face, T)`` and ``cells()`` -- the
engine's `Engine`, or the oracle's CPU reference for the same problem.
"""
import numpy as np

from . import problems as P
from .units import UNITS


def marshak_l1(x, t_gas, ref):
    """ComputeL1 with useGas (MarshakCommon.hpp:193-228): walk the reference
    points in order, interpolate the simulated profile linearly at each, and
    average |T_sim - T_ref| / T_ref over the points whose T_ref exceeds 1e-4
    keV; stop at the first point past the last simulated interval.  `x` and
    `t_gas` are sorted by x; `ref` is the (n, 3) table x, T_gas, T_rad [K].
    Returns -1 when nothing was compared."""
    keV = UNITS["kev_kelvin"]
    l1, count, j = 0.0, 0, 0
    n = len(x)
    if n == 0 or len(ref) == 0:
        return -1.0
    for rx, rt in zip(ref[:, 0], ref[:, 1]):
        while j + 1 < n and x[j + 1] < rx:
            j += 1
        if j + 1 >= n:
            break
        frac = (rx - x[j]) / (x[j + 1] - x[j])
        sim = (t_gas[j] + frac * (t_gas[j + 1] - t_gas[j])) / keV
        r = rt / keV
        if r > 1e-4:
            l1 += abs(sim - r) / r
            count += 1
    return l1 / count if count else -1.0


def densmore_l1(x, t_gas, ref):
    """The Densmore example's L1 (examples/densmore2012/main.cpp:323-343): for
    each reference point (x [cm], T [keV]) the simulated profile is
    interpolated linearly (points past the last simulated interval are
    skipped) and |T_sim - T_ref| in keV is averaged."""
    keV = UNITS["kev_kelvin"]
    l1, count = 0.0, 0
    n = len(x)
    for rx, rt in zip(ref[:, 0], ref[:, 1]):
        j = 0
        while j + 1 < n and x[j + 1] < rx:
            j += 1
        if j + 1 >= n:
            continue
        frac = (rx - x[j]) / (x[j + 1] - x[j])
        sim = (t_gas[j] + frac * (t_gas[j + 1] - t_gas[j])) / keV
        l1 += abs(sim - rt)
        count += 1
    return l1 / count if count else -1.0


def _profile(problem, cells):
    xc, _, _ = problem.cell_centers()
    order = np.argsort(xc, kind="stable")
    t_rad = np.power(np.maximum(cells["erad_time_avg"], 0.0) / UNITS["arad"], 0.25)
    return xc[order], cells["temperature"][order], t_rad[order]


def marshak_schedule(problem):
    """The example's (t_now, dt) sequence (MarshakCommon.hpp:331-351): dt starts
    at the initial step, is clipped to the time left, and after each step
    becomes min(max(initial, t * 1e-3), 5e-11)."""
    q = P.MARSHAK_PARAMS[problem]
    dt0, tf = q["initial_dt"], P.MARSHAK_FINAL_TIME
    t, dt = 0.0, dt0
    while t < tf:
        t_now = max(t, dt0)
        dt = min(dt, tf - t)
        yield t_now, dt
        t += dt
        dt = min(max(dt0, t * 1e-3), 5e-11)


def run_marshak_wave(make, problem=1, **kw):
    """Run Marshak wave `problem` to 1 ns: before every step the bath on x=0 is
    set to BathTemperature(max(t, dt0)).  Returns x, T_gas, T_rad (sorted by
    x, T_rad from the time-averaged radiation energy density) and the step count."""
    p = P.marshak_wave(problem, **kw)
    eng = make(p)
    steps = 0
    try:
        for t_now, dt in marshak_schedule(problem):
            eng.set_face_temperature(0, P.marshak_bath_temperature(problem, t_now))
            eng.step(dt)
            steps += 1
        x, tg, tr = _profile(p, eng.cells())
    finally:
        eng.close()
    return {"x": x, "t_gas": tg, "t_rad": tr, "steps": steps}


def run_densmore2012(make, steps=200, **kw):
    """Run the Densmore benchmark: `steps` steps of 5 ps (200 reach 1 ns)."""
    p = P.densmore2012(**kw)
    eng = make(p)
    try:
        for _ in range(steps):
            eng.step(p.dt)
        x, tg, tr = _profile(p, eng.cells())
    finally:
        eng.close()
    return {"x": x, "t_gas": tg, "t_rad": tr, "steps": steps}
