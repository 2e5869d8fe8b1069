#!/usr/bin/env python
"""Benchmark: particle-segments/s of the IMC time step on the 64^3 two-material
step-opacity cube (Random Walk where kappa*dx > 10, ~1e7 source packets per
step, comb to ~1e7 census), one B200 per rank.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl storm|reference]

A step is one full IMC time step: emission, transport to census, comb, material
update.  `value` = segments of all ranks / max-over-ranks device time of the K
timed steps (CUDA events on the engine's stream); inputs (the ~1 GB particle
bank) are far larger than L2.  `e2e` is the same metric through the C ABI with
the census copied host->device from pinned memory before each step and the
census plus material temperatures copied back after it.  The reference arm
times the reference's own serial path (compiled from its sources, or the
oracle port where that build is absent) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-segments/s FP32-track vs FP64 on 1 B200 at stated sigma; p50/p99 step latency"
UNIT = "segments/s"
# Algorithmic bytes per segment of the FP64 form: particle state read + write
# (2 x 72 B), cell sigma_a and Fleck factor (16 B), two tallies (16 B).
BYTES_PER_SEGMENT_FP64 = 176
# FP32-tracking form: state 2 x 44 B (cell 4, offset 3x4, direction 3x4, weight 8,
# time 8), cell constants 16 B, tallies 16 B.
BYTES_PER_SEGMENT_FP32 = 120


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="storm", choices=["storm", "reference"])
    ap.add_argument("--n", type=int, default=64, help="cells per axis")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--dev-seeds", type=int, default=8, help="seeds per form of the FP32-vs-FP64 deviation study")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--segments-per-visit", type=int, default=0)
    ap.add_argument("--min-blocks", type=int, default=0, help="transport occupancy variant (1-4)")
    ap.add_argument("--waves", type=int, default=4)
    ap.add_argument("--refill", type=int, default=-1, help="1 persistent refill kernel, 0 bank visits")
    ap.add_argument("--burst", type=int, default=8)
    ap.add_argument("--mg-steps", type=int, default=5, help="timed steps of the multigroup run (0 = skip it)")
    ap.add_argument("--voronoi-steps", type=int, default=5, help="timed steps of the Voronoi-mesh run (0 = skip it)")
    ap.add_argument("--voronoi-cells", type=int, default=200000)
    ap.add_argument("--voronoi-packets", type=float, default=2e7, help="packets per step of the Voronoi-mesh run")
    ap.add_argument("--mg-n", type=int, default=128)
    ap.add_argument("--serving-requests", type=int, default=32, help="requests in the serving run (0 = skip it)")
    ap.add_argument("--serving-slots", type=int, default=6)
    ap.add_argument("--serving-workers", type=int, default=3)
    return ap.parse_args()


def workload(n=64, seed=42):
    from storm_b200 import problems
    # 3 photons per cell and 450 packets per x=0 boundary face: ~1e7 source
    # packets per step; comb to Ncells * 20 * 2 ~ 1.05e7 census particles.
    return problems.step_cube(n=n, new_photons_per_cell=3, face_packets=450, comb_nmin=20, comb_factor=2.0,
                              seed=seed, dt=1e-11)


def workload_config(n):
    """The workload both arms report (identical dicts): what each arm computes
    it in, and on how many processes, is stated outside `config`."""
    return {"workload": f"step_cube {n}^3 gray IMC, kappa_a=1|1000 1/cm, RW kappa*dx>10, dt=1e-11 s, "
                        f"3 photons/cell + 450/face source, comb Nmin=20 factor=2",
            "cells": n ** 3, "packets_per_step": "~1e7", "census_per_step": "~1e7",
            "l2": "inputs larger than L2 (particle bank ~1 GB)"}


# ---------------------------------------------------------------------- clocks
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, v in zip(names, r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------- distributed
def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "storm" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local, dist


def reduce(dist, value, op, impl):
    if dist is None:
        return value
    import torch
    dev = "cuda" if impl == "storm" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist, impl):
    if dist is None:
        return
    import torch
    if impl == "storm":
        dist.barrier(device_ids=[torch.cuda.current_device()])
    else:
        dist.barrier()


# ---------------------------------------------------------------------- CPU baseline
def _ref_worker(q):
    """One bounded sample of the bench's own workload (the same cube, packet
    densities and comb as `workload`) on the reference's serial path: `steps`
    IMC steps from the initial state, the last `timed` of them timed (the
    manager's own step wall time)."""
    seed, steps, timed, use_ref, n = q
    sys.path.insert(0, ROOT)
    p = workload(n, seed=seed)
    if use_ref:
        from oracle import ref
        m = ref.Reference(p)
        segs, wall = 0, 0.0
        for s in range(steps):
            o = m.step()
            if s >= steps - timed:
                segs += o["segments"]
                wall += o["wall_seconds"]
        m.close()
        return segs, wall
    from oracle import orc
    m = orc.Oracle(p)
    segs, wall = 0, 0.0
    for s in range(steps):
        t = time.perf_counter()
        st = m.step()
        dt = time.perf_counter() - t
        if s >= steps - timed:
            segs += st["segments"]
            wall += dt
    return segs, wall


def cpu_baseline(n, cores, steps=1, timed=1):
    """The reference's serial path on `cores` independent processes (one core
    each), each running `steps` IMC steps of the bench's workload and timing the
    last `timed`.  Rate = all processes' segments / the slowest process's time."""
    from oracle import ref, orc
    use_ref = ref.available()
    if not use_ref and not os.path.exists(orc.LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    jobs = [(1000 + k, steps, timed, use_ref, n) for k in range(cores)]
    if cores == 1:
        res = [_ref_worker(jobs[0])]
    else:
        with ctx.Pool(cores, maxtasksperchild=1) as pool:
            res = pool.map(_ref_worker, jobs)
    segs = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    which = "IMC step 1 (from the initial state)" if steps == 1 else \
        f"IMC step{'s' if timed > 1 else ''} {steps - timed + 1}-{steps} after {steps - timed} untimed"
    return {"value": segs / wall, "unit": UNIT, "cores": cores, "kind": "reference" if use_ref else "port",
            "sample": f"{cores} process(es), one core each, {which} of the bench workload ({workload_config(n)['workload']}); "
                      f"{segs} segments in {wall:.1f} s"}


# ---------------------------------------------------------------------- storm arm
def _peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        v = json.load(open(path)).get("hbm_gbs")
        if v:
            return float(v), "measured"
    return 6650.0, "fallback"


def run_form(args, precision, seed, local, dist, timed=True):
    """Warm up, then time args.steps IMC steps of one form; returns its numbers."""
    import torch
    from storm_b200.engine import Engine
    p = workload(args.n, seed=seed)
    p.device = local
    p.precision = precision
    p.per_cell_segment_counters = False
    eng = Engine(p)
    if args.segments_per_visit:
        eng.set_segments_per_visit(args.segments_per_visit)
    if args.min_blocks:
        eng.set_transport_variant(args.min_blocks, args.waves)
    if args.refill >= 0:
        eng.set_transport_mode(bool(args.refill), args.burst)
    eng.set_profiling(True)
    for _ in range(args.warmup):
        eng.step()
    torch.cuda.synchronize()
    barrier(dist, "storm")
    eng.transport_timing(reset=True)
    l0 = eng.launches()
    step_ms, segs = [], 0
    phase = {"emit": 0.0, "transport": 0.0, "comb": 0.0}
    for _ in range(args.steps if timed else 0):
        st = eng.step()
        step_ms.append(st["step_ms"])
        segs += st["segments"]
        for k in phase:
            phase[k] += st[k + "_ms"]
    torch.cuda.synchronize()
    barrier(dist, "storm")
    k = max(len(step_ms), 1)
    phase = {name: v / k for name, v in phase.items()}
    phase["other"] = sum(step_ms) / k - sum(phase.values())
    out = {"engine": eng, "problem": p, "step_ms": step_ms, "segments": segs, "launches": eng.launches() - l0,
           "transport": eng.transport_timing(reset=True), "phase_ms": phase}
    return out


def transport_kernel(args, fp32):
    """Name of the transport kernel the run launches (refill is the engine default;
    the gray FP32 form without the DDMC branch, Form32T<false, false>, for this
    workload)."""
    form = "Form32Lean" if fp32 else "Form64"
    if args.refill != 0:
        return f"k_transport_refill<{form}>"
    return "k_transport32" if fp32 else "k_transport"


def measured_traffic(kernel):
    """DRAM bytes per segment of `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "transport_traffic.json")
    if not os.path.exists(path):
        return None, None
    entry = json.load(open(path)).get(kernel)
    if not entry:
        return None, None
    return entry["dram_bytes_per_segment"], entry["capture"]


def measured_issue(kernel):
    """Warp instructions and thread instructions per segment of `kernel` from
    the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "transport_issue.json")
    if not os.path.exists(path):
        return None
    return json.load(open(path)).get(kernel)


def roofline(res, bytes_per_segment, kernel, sm_mhz=None):
    """The HBM roofline of the transport kernel by the fixed per-segment byte
    convention, with the measured DRAM traffic beside it, and a second,
    issue-based fraction: warp instructions per segment (ncu) x segments/s
    against 148 SMs x 4 schedulers x the SM clock sampled in the timed region,
    with the active lanes per warp instruction."""
    peak, src = _peak()
    tt = res["transport"]
    mean_ms = tt["kernel_ms"] / max(tt["launches"], 1)
    segs_per_launch = tt["segments"] / max(tt["launches"], 1)
    bytes_per_launch = bytes_per_segment * segs_per_launch
    achieved = bytes_per_launch / (mean_ms / 1000.0) / 1e9
    per_seg, capture = measured_traffic(kernel)
    traffic = per_seg * segs_per_launch if per_seg is not None else None
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "traffic": traffic, "kernel": kernel, "bytes_per_segment": bytes_per_segment,
           "mean_launch_ms": mean_ms, "launches": tt["launches"], "segments_per_launch": segs_per_launch,
           "peak_source": src, "note": "peak = measured copy bandwidth (" + src + ")"}
    if capture:
        out["traffic_source"] = capture
    if per_seg is not None:
        out["dram_frac"] = traffic / (mean_ms / 1000.0) / 1e9 / peak   # measured bytes against the peak
    iss = measured_issue(kernel)
    if iss:
        clock = (sm_mhz or 1965.0) * 1e6
        seg_rate = segs_per_launch / (mean_ms / 1000.0)
        inst_rate = iss["warp_inst_per_segment"] * seg_rate
        out["issue"] = {"warp_inst_per_segment": iss["warp_inst_per_segment"],
                        "achieved_inst_per_s": inst_rate, "peak_inst_per_s": 148 * 4 * clock,
                        "frac": inst_rate / (148 * 4 * clock),
                        "lanes_active_per_inst": iss["thread_inst_per_segment"] / iss["warp_inst_per_segment"],
                        "sm_mhz": clock / 1e6, "source": iss["capture"]}
    return out


def e2e_run(args, eng, p, dist):
    """The same metric through the C ABI with host buffers, as a caller of the
    drop-in runs it: each step takes the census from page-locked host memory
    and returns the new census there (storm_cuda_step_host, which overlaps the
    upload with the step's work that does not need the census), and the
    material temperatures come back after it.  The census travels with the
    fields a step reads (position, direction, weight, cell) both ways; time
    left and initial weight, which every step sets for its census at its start,
    are neither sent nor read back."""
    import torch
    from storm_b200.engine import Particles
    import numpy as np
    n = eng.census_count()
    bufs = [Particles.pinned(max(2 * n, 1)) for _ in range(2)]
    for b in bufs:
        b.time_left = b.initial_weight = None
    pin_T = torch.empty(p.ncells, dtype=torch.float64, pin_memory=True).numpy()
    host = eng.census(out=bufs[0])
    rec = 7 * 8 + 4    # position, direction, weight, cell
    torch.cuda.synchronize()
    barrier(dist, "storm")
    t0 = time.perf_counter()
    segs, h2d, d2h, done = 0, 0, 0, 0
    for k in range(args.e2e_steps):
        if eng.census_count() > bufs[0].n:
            break
        st, out = eng.step_host(host, bufs[(k + 1) % 2])
        h2d += host.n * rec
        segs += st["segments"]
        d2h += out.n * rec
        eng.temperature(out=pin_T)
        d2h += p.ncells * 8
        host = out
        done += 1
    torch.cuda.synchronize()
    wall = reduce(dist, time.perf_counter() - t0, "max", "storm")
    allsegs = reduce(dist, segs, "sum", "storm")
    link = link_bandwidth()
    steps = max(done, 1)
    floor_ms = (h2d / steps) / link["h2d_gbs"] / 1e6 + (d2h / steps) / link["d2h_gbs"] / 1e6
    return {"value": allsegs / wall, "unit": UNIT, "h2d_bytes_per_step": int(h2d / steps),
            "d2h_bytes_per_step": int(d2h / steps), "steps": done,
            "ms_per_step": wall / steps * 1e3, "link": link, "copy_ms_per_step_at_link_rate": floor_ms,
            "note": "census in and out through storm_cuda_step_host (upload overlapped with the prestep, the "
                    "emission and the new packets' transport), without time left and initial weight, which "
                    "the step sets; temperatures through storm_cuda_get_cell_arrays; page-locked host buffers; "
                    "copies and host-side checks inside the timed region (wall clock); link = one 1 GiB "
                    "page-locked copy each way, CUDA-event timed"}


def link_bandwidth(nbytes=1 << 30):
    """Host<->device copy rate of this GPU's link: one page-locked copy of
    `nbytes` each way after a warm-up copy, timed with CUDA events."""
    import torch
    host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    dev = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    out = {}
    for name, (dst, src) in (("h2d_gbs", (dev, host)), ("d2h_gbs", (host, dev))):
        dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        dst.copy_(src, non_blocking=True)
        b.record()
        torch.cuda.synchronize()
        out[name] = nbytes / (a.elapsed_time(b) * 1e-3) / 1e9
    del host, dev
    return out


def kernel_roofline(kernel, segs, ms_per_step, steps, sm_mhz=None):
    """A transport kernel against its binding ceiling: ncu's warp instructions
    per segment (profiles/transport_issue.json) times the kernel's segments/s,
    against 148 SMs x 4 schedulers x the SM clock, and its measured DRAM bytes
    per segment against the copy bandwidth."""
    rate = segs / steps / (ms_per_step / 1e3) if ms_per_step > 0 else 0.0
    out = {"kernel": kernel, "kernel_ms_per_step": ms_per_step, "segments_per_s_in_kernel": rate}
    iss = measured_issue(kernel)
    if iss and rate:
        clock = (sm_mhz or 1965.0) * 1e6
        out["issue"] = {"warp_inst_per_segment": iss["warp_inst_per_segment"],
                        "frac": iss["warp_inst_per_segment"] * rate / (148 * 4 * clock),
                        "lanes_active_per_inst": iss["thread_inst_per_segment"] / iss["warp_inst_per_segment"],
                        "sm_mhz": clock / 1e6, "source": iss["capture"]}
    per_seg, capture = measured_traffic(kernel)
    if per_seg is not None and rate:
        peak, src = _peak()
        out["dram"] = {"bytes_per_segment": per_seg, "achieved_gbs": per_seg * rate / 1e9,
                       "frac": per_seg * rate / 1e9 / peak, "peak_gbs": peak, "peak_source": src, "source": capture}
    return out


def mg_run(args, sm_mhz=None):
    """The multigroup configuration: a 128^3 unit cube, 64 groups log-spaced over
    [0.01, 100] keV, kappa_g = 100 nu_g^-3 (1 - exp(-nu_g/T)) cm^-1, initial T
    uniform in [0.01, 0.1] keV per cell (seeded), cell emission from the
    Planck-weighted opacity spectrum (about 4e7 packets per step at 2 packets
    per cell), comb Nmin=12 factor=2, PGRW.  Both forms on the same problem;
    device-timed steps after 2 warm-up steps."""
    import numpy as np
    from storm_b200 import _abi as A
    from storm_b200 import problems
    from storm_b200.engine import Engine
    out = {"workload": f"mg_cube {args.mg_n}^3, 64 groups [0.01,100] keV, kappa0=100 nu^-3 (1-exp(-nu/T)), "
                       "T0 U[0.01,0.1] keV, 2 photons/cell base allocation, comb Nmin=12 factor=2, PGRW",
           "steps": args.mg_steps}
    temps = {}
    for name, prec in (("fp32", A.PRECISION_FP32_TRACK), ("fp64", A.PRECISION_FP64)):
        p = problems.mg_cube(n=args.mg_n, groups=64, kappa0=100.0, new_photons_per_cell=2, comb_nmin=12, seed=3,
                             precision=prec)
        p.per_cell_segment_counters = False
        e = Engine(p)
        e.set_profiling(True)   # the transport kernel's own CUDA-event time
        for _ in range(2):
            e.step()
        segs, ms, tms, lat = 0, 0.0, 0.0, []
        for _ in range(args.mg_steps):
            st = e.step()
            segs += st["segments"]
            ms += st["step_ms"]
            tms += st["transport_ms"]
            lat.append(st["step_ms"])
        out[name] = {"segments_per_s": segs / (ms / 1e3), "ms_per_step": ms / args.mg_steps,
                     "segments_per_step": segs / args.mg_steps, "emitted_per_step": st["emitted_cells"],
                     "census_per_step": st["census_out"], "step_ms_p99": float(np.percentile(lat, 99)),
                     "device_gb": e.memory_bytes() / 1e9,
                     "transport": kernel_roofline("k_transport_refill<Form32MGLean>" if name == "fp32" else
                                                  "k_transport_refill<Form64MG>", segs, tms / args.mg_steps,
                                                  args.mg_steps, sm_mhz)}
        temps[name] = e.cells()["temperature"]
        e.close()
    out["fp32_over_fp64"] = out["fp32"]["segments_per_s"] / out["fp64"]["segments_per_s"]
    out["mean_relative_temperature_difference"] = float(np.mean(np.abs(temps["fp32"] - temps["fp64"]) / temps["fp64"]))
    return out


def voronoi_run(args, sm_mhz=None):
    """Gray IMC on a Voronoi mesh of 2e5 seeded uniform generators in the unit
    cube (about 15 faces per cell; the engine's own builder), per-cell
    lognormal opacity (median 10 1/cm, sigma_ln 1), lognormal initial
    temperature (median 0.05 keV), about 2e7 packets per step, Random Walk.
    Both forms on the same mesh; device-timed steps after 2 warm-up steps."""
    import numpy as np
    from storm_b200 import _abi as A
    from storm_b200 import problems
    from storm_b200.engine import Engine
    from storm_b200.mesh import build_voronoi
    t0 = time.perf_counter()
    mesh = build_voronoi(np.random.default_rng(5).random((args.voronoi_cells, 3)) * (1 - 2e-9) + 1e-9)
    build_s = time.perf_counter() - t0
    out = {"workload": f"Voronoi mesh of {args.voronoi_cells} cells in the unit cube "
                       f"({mesh.cell_faces.size / mesh.ncells:.1f} faces/cell), kappa lognormal median 10 1/cm "
                       f"sigma_ln 1, T0 lognormal median 0.05 keV, ~{args.voronoi_packets:.0e} packets/step, "
                       "vacuum box, RW",
           "steps": args.voronoi_steps, "mesh_build_s": build_s}
    temps = {}
    for name, prec in (("fp32", A.PRECISION_FP32_TRACK), ("fp64", A.PRECISION_FP64)):
        p = problems.voronoi_cube(ncells=args.voronoi_cells, packets_per_step=args.voronoi_packets, seed=5, mesh=mesh,
                                  precision=prec)
        p.per_cell_segment_counters = False
        e = Engine(p)
        e.set_profiling(True)   # the transport kernel's own CUDA-event time
        for _ in range(2):
            e.step()
        segs, ms, tms, lat = 0, 0.0, 0.0, []
        for _ in range(args.voronoi_steps):
            st = e.step()
            segs += st["segments"]
            ms += st["step_ms"]
            tms += st["transport_ms"]
            lat.append(st["step_ms"])
        out[name] = {"segments_per_s": segs / (ms / 1e3), "ms_per_step": ms / args.voronoi_steps,
                     "segments_per_step": segs / args.voronoi_steps, "emitted_per_step": st["emitted_cells"],
                     "census_per_step": st["census_out"], "step_ms_p99": float(np.percentile(lat, 99)),
                     "device_gb": e.memory_bytes() / 1e9,
                     "transport": kernel_roofline("k_transport_refill<Form32Poly>" if name == "fp32" else
                                                  "k_transport_refill<Form64Poly>", segs,
                                                  tms / args.voronoi_steps, args.voronoi_steps, sm_mhz)}
        temps[name] = e.cells()["temperature"]
        e.close()
    out["fp32_over_fp64"] = out["fp32"]["segments_per_s"] / out["fp64"]["segments_per_s"]
    out["mean_relative_temperature_difference"] = float(np.mean(np.abs(temps["fp32"] - temps["fp64"]) / temps["fp64"]))
    return out


def serving_run(args):
    """Many independent FP32-tracking problems (N log-uniform in [16, 48],
    1e4-1e6 packets/step log-uniform, kappa uniform in [0.1, 1000], 5-20 steps)
    through the serving loop, against the same requests one at a time.  The
    concurrent run receives the requests as a Poisson stream at 4x the rate the
    one-at-a-time server completes them.  One untimed pass first fills the
    engine's device memory cache, as a long-running server's would be.  Both
    arms run three times, alternating; each reports its median run (by wall
    time) and the ratios are taken between the medians."""
    import numpy as np
    from storm_b200 import problems
    from storm_b200.engine import Server
    mix = problems.serving_mix(args.serving_requests, seed=11)

    def run(slots, workers, gaps):
        srv = Server(max_active=slots, workers=workers)
        t0 = time.perf_counter()
        for (p, steps), gap in zip(mix, gaps):
            if gap > 0:
                time.sleep(gap)
            srv.submit(p, steps, want_temperature=False)
        srv.drain()
        wall = time.perf_counter() - t0
        st = srv.stats()
        res = srv.poll()
        srv.close()
        ok = sum(1 for r in res if r["status"] == 0)
        return {"segments_per_s": st["segments"] / wall, "wall_s": wall, "segments": st["segments"],
                "step_ms_p50": st["step_ms_p50"], "step_ms_p99": st["step_ms_p99"], "completed": ok,
                "queued_ms_max": max((r["queued_ms"] for r in res), default=0.0),
                "peak_device_gb": st["peak_device_bytes"] / 1e9, "slots": slots, "workers": workers}

    def median_run(runs):
        runs = sorted(runs, key=lambda r: r["wall_s"])
        out = dict(runs[len(runs) // 2])
        out["wall_s_runs"] = [round(r["wall_s"], 4) for r in runs]
        return out

    run(args.serving_slots, args.serving_workers, [0.0] * len(mix))   # warm the device memory cache
    alone_runs = [run(1, 1, [0.0] * len(mix))]
    rng = np.random.default_rng(12)
    mean_gap = alone_runs[0]["wall_s"] / len(mix) / 4.0
    gaps = [0.0] + list(rng.exponential(mean_gap, len(mix) - 1))
    mixed_runs = [run(args.serving_slots, args.serving_workers, gaps)]
    for _ in range(2):
        alone_runs.append(run(1, 1, [0.0] * len(mix)))
        mixed_runs.append(run(args.serving_slots, args.serving_workers, gaps))
    alone, mixed = median_run(alone_runs), median_run(mixed_runs)
    return {"requests": len(mix), "form": "fp32-track",
            "mix": "uniform cubes, N log-uniform [16,48], packets/step log-uniform [1e4,1e6], "
                   "kappa uniform [0.1,1000] 1/cm, 5-20 steps, seeded",
            "one_at_a_time": alone, "concurrent": mixed,
            "throughput_ratio": mixed["segments_per_s"] / max(alone["segments_per_s"], 1e-300),
            "p99_step_latency_ratio": mixed["step_ms_p99"] / max(alone["step_ms_p99"], 1e-300),
            "arrivals": f"Poisson, mean gap {mean_gap * 1e3:.2f} ms (4x the one-at-a-time completion rate)"}


def run_storm(args, ws, rank, local, dist):
    import numpy as np
    import torch
    from storm_b200 import _abi as A
    torch.cuda.set_device(local)
    seed = 42 + rank
    clocks = Clocks(local)
    clocks.start()
    f32 = run_form(args, A.PRECISION_FP32_TRACK, seed, local, dist)
    f64 = run_form(args, A.PRECISION_FP64, seed, local, dist)
    ck = clocks.stop()

    def rate(res):
        ms = reduce(dist, sum(res["step_ms"]), "max", "storm")
        sg = reduce(dist, res["segments"], "sum", "storm")
        return sg / (ms / 1000.0), ms

    v32, ms32 = rate(f32)
    v64, ms64 = rate(f64)
    f32["engine"].close()
    f64["engine"].close()
    dev = deviation_study(args, local) if (rank == 0 and args.dev_seeds > 1) else None
    e2e = None
    if args.e2e_steps > 0:
        from storm_b200.engine import Engine
        p = workload(args.n, seed=seed)
        p.device, p.precision, p.per_cell_segment_counters = local, A.PRECISION_FP32_TRACK, False
        eng = Engine(p)
        for _ in range(args.warmup):
            eng.step()
        e2e = e2e_run(args, eng, p, dist)
        eng.close()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.n, 1, steps=1, timed=1)
    serving = serving_run(args) if (rank == 0 and ws == 1 and args.serving_requests > 0) else None
    multigroup = mg_run(args, (ck or {}).get("sm_mhz")) if (rank == 0 and ws == 1 and args.mg_steps > 0) else None
    voronoi = voronoi_run(args, (ck or {}).get("sm_mhz")) if (rank == 0 and ws == 1 and args.voronoi_steps > 0) else None
    if rank == 0:
        lat = sorted(f32["step_ms"])
        line = {
            "metric": METRIC, "value": v32, "fp64_value": v64, "fp32_over_fp64": v32 / v64, "unit": UNIT,
            "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-track/f64-tally",
            "form": "value: FP32 cell-local tracking with FP64 time, weights and tallies; "
                    "fp64_value: the all-FP64 form on the same workload",
            "parallelism": f"{ws} independent problem(s), one per GPU",
            "data": "synthetic (seeded Philox streams)",
            "config": workload_config(args.n),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "segments_per_step": f32["segments"] / args.steps,
            "phase_ms_per_step": f32["phase_ms"],
            "roofline": roofline(f32, BYTES_PER_SEGMENT_FP32, transport_kernel(args, True),
                                 ck["sm_mhz"] if ck else None),
            "fp64": {"value": v64, "ms_per_step": ms64 / args.steps, "dtype": "f64",
                     "latency_ms": {"p50": float(np.percentile(f64["step_ms"], 50)),
                                    "p99": float(np.percentile(f64["step_ms"], 99))},
                     "segments_per_step": f64["segments"] / args.steps,
                     "phase_ms_per_step": f64["phase_ms"],
                     "roofline": roofline(f64, BYTES_PER_SEGMENT_FP64, transport_kernel(args, False),
                                          ck["sm_mhz"] if ck else None)},
            "fp32_vs_fp64_deviation": dev,
            "cpu_baseline": cpu, "e2e": e2e, "serving": serving, "multigroup": multigroup, "voronoi": voronoi, "clocks": ck,
            "gpu_launches": f32["launches"],
            "transport_share": f32["transport"]["kernel_ms"] / max(sum(f32["step_ms"]), 1e-9),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def deviation_study(args, local):
    """The FP32-tracking form's deviation from the FP64 form, in units of the
    batch-estimated statistical error.  Both forms run the bench workload
    (warm-up + timed step count) on `dev_seeds` independent seeds each; a second
    FP64 batch on a third set of seeds is the control.
    Per cell and per quantity (material temperature, the last step's deposit,
    time-averaged and census radiation energy) the difference of batch means is
    a Welch z (storm_b200.batchstats); reported: the fraction of populated
    cells within 1, 2 and 3 sigma, the largest |z| against its Bonferroni
    bound, and the same for FP64 against FP64."""
    import numpy as np
    from storm_b200 import _abi as A
    from storm_b200 import batchstats
    from storm_b200.engine import Engine
    steps = args.warmup + args.steps

    def batch(precision, seeds):
        out = []
        for s in seeds:
            p = workload(args.n, seed=s)
            p.device, p.precision, p.per_cell_segment_counters = local, precision, False
            e = Engine(p)
            out.append(batchstats.run_snapshots(e, p, steps, (steps,)))
            e.close()
        return np.array(out)

    k = args.dev_seeds
    r32 = batch(A.PRECISION_FP32_TRACK, range(42, 42 + k))
    r64 = batch(A.PRECISION_FP64, range(1042, 1042 + k))
    r64b = batch(A.PRECISION_FP64, range(2042, 2042 + k))

    def summary(res):
        g = res["all"]
        return {"tests": g["tests"], "frac_within": g["frac_within"], "max_abs_z": g["max_abs_z"],
                "z_bound": g["z_bound"], "above_3": g["above_threshold"], "k_max": g["k_max"],
                "mean_z": g["mean_z"], "rms_z": g["rms_z"], "totals_max_abs_z": res["totals"]["max_abs_z"],
                "passed": res["passed"],
                "per_quantity_frac_within_1": {q: res[q]["frac_within"]["1"] for q in batchstats.QUANTITIES}}
    fp32 = summary(batchstats.compare(r32, r64))
    ctrl = summary(batchstats.compare(r64b, r64))
    return {"seeds_per_form": args.dev_seeds, "steps": steps,
            "quantities": list(batchstats.QUANTITIES),
            "z": "Welch z of the per-cell batch means (normal-equivalent), FP32 vs FP64 on independent seeds",
            "fp32_vs_fp64": fp32, "fp64_vs_fp64_control": ctrl,
            "within_1_sigma_like_fp64": bool(fp32["frac_within"]["1"] >= ctrl["frac_within"]["1"] - 0.05),
            "statement": "FP32 differs from FP64 by no more than FP64 differs from itself over independent seeds"
                         if fp32["passed"] else "FP32 deviates beyond the statistical error of the FP64 form"}


# ---------------------------------------------------------------------- reference arm
# host memory one reference process holds through IMC step 2 of the 64^3 workload
REF_PROCESS_BYTES = 9e9


def run_reference(args, ws, rank, dist):
    """The reference's serial path on the bench's exact workload: one process
    per host core (as many as host memory holds), each running the untimed IMC
    step 1 and the timed IMC step 2 -- bounded by steps, not by packet
    density, so that the whole arm takes a couple of minutes whatever
    --steps / --warmup say."""
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    cores = os.cpu_count() or 1
    per_process = REF_PROCESS_BYTES * (args.n / 64.0) ** 3
    try:
        import psutil
        cores = max(1, min(cores, int(psutil.virtual_memory().available * 0.8 / per_process)))
    except ImportError:
        pass
    res = cpu_baseline(args.n, cores, steps=2, timed=1)
    value = res["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded std::mt19937_64 in the reference)",
            "form": "the reference's serial FP64 path (MonteCarloManagerSerial + RadiationIMC + CombPopulationControl)",
            "parallelism": f"{cores} independent reference processes, one host core each",
            "config": workload_config(args.n),
            "cpu_baseline": res | {"value": value},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    ws, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, ws, rank, dist)
    else:
        run_storm(args, ws, rank, local, dist)


if __name__ == "__main__":
    main()
