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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="storm", choices=["storm", "reference"])
    ap.add_argument("--n", type=int, default=64, help="cells per axis")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--segments-per-visit", type=int, default=0)
    ap.add_argument("--min-blocks", type=int, default=0, help="transport occupancy variant (1-4)")
    ap.add_argument("--waves", type=int, default=4)
    return ap.parse_args()


def workload(n=64, seed=42):
    from storm_b200 import problems
    # 3 photons per cell and 450 packets per x=0 boundary face: ~1e7 source
    # packets per step; comb to Ncells * 20 * 2 ~ 1.05e7 census particles.
    return problems.step_cube(n=n, new_photons_per_cell=3, face_packets=450, comb_nmin=20, comb_factor=2.0,
                              seed=seed, dt=1e-11)


def workload_config(n):
    return {"workload": f"step_cube {n}^3 gray IMC, kappa_a=1|1000 1/cm, RW kappa*dx>10, dt=1e-11 s, "
                        f"3 photons/cell + 450/face source, comb Nmin=20 factor=2",
            "cells": n ** 3, "packets_per_step": "~1e7", "census_per_step": "~1e7",
            "l2": "inputs larger than L2 (particle bank ~1 GB)", "precision": "fp64"}


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
    """One bounded sample of the workload on the reference's serial path:
    3 time steps of the same 64^3 cube at 1 photon per cell (2.7e6 packets/step)
    and 30 per boundary face; the last 2 steps are timed."""
    seed, steps, use_ref, n = q
    sys.path.insert(0, ROOT)
    from storm_b200 import problems
    p = problems.step_cube(n=n, new_photons_per_cell=1, face_packets=30, comb_nmin=2, comb_factor=2.0, seed=seed)
    if use_ref:
        from oracle import ref
        m = ref.Reference(p)
        segs, wall = 0, 0.0
        for s in range(steps):
            o = m.step()
            if s > 0:
                segs += o["segments"]
                wall += o["wall_seconds"]
        return segs, wall
    from oracle import orc
    m = orc.Oracle(p)
    segs, wall = 0, 0.0
    for s in range(steps):
        t = time.perf_counter()
        st = m.step()
        dt = time.perf_counter() - t
        if s > 0:
            segs += st["segments"]
            wall += dt
    return segs, wall


def cpu_baseline(n, cores, steps=3):
    from oracle import ref, orc
    use_ref = ref.available()
    if not use_ref and not os.path.exists(orc.LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    jobs = [(1000 + k, steps, use_ref, n) for k in range(cores)]
    if cores == 1:
        res = [_ref_worker(jobs[0])]
    else:
        with ctx.Pool(cores) as pool:
            res = pool.map(_ref_worker, jobs)
    segs = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    return {"value": segs / wall, "unit": UNIT, "cores": cores, "kind": "reference" if use_ref else "port",
            "sample": f"{cores} process(es) x {steps - 1} timed IMC steps of the {n}^3 cube at 1 photon/cell "
                      f"(2.7e6 packets/step), 30/face, comb Nmin=2; {segs} segments in {wall:.1f} s"}


# ---------------------------------------------------------------------- storm arm
def run_storm(args, ws, rank, local, dist):
    import numpy as np
    import torch
    from storm_b200.engine import Engine, Particles
    torch.cuda.set_device(local)
    p = workload(args.n, seed=42 + rank)
    p.device = local
    p.per_cell_segment_counters = False
    eng = Engine(p)
    if args.segments_per_visit:
        eng.set_segments_per_visit(args.segments_per_visit)
    if args.min_blocks:
        eng.set_transport_variant(args.min_blocks, args.waves)
    eng.set_profiling(True)
    for _ in range(args.warmup):
        eng.step()
    torch.cuda.synchronize()
    barrier(dist, "storm")
    clocks = Clocks(local)
    clocks.start()
    eng.transport_timing(reset=True)
    l0 = eng.launches()
    step_ms, segs = [], 0
    for _ in range(args.steps):
        st = eng.step()
        step_ms.append(st["step_ms"])
        segs += st["segments"]
    torch.cuda.synchronize()
    barrier(dist, "storm")
    ck = clocks.stop()
    launches = eng.launches() - l0
    tt = eng.transport_timing(reset=True)
    total_ms = reduce(dist, sum(step_ms), "max", "storm")
    all_segs = reduce(dist, segs, "sum", "storm")
    value = all_segs / (total_ms / 1000.0)

    # dominant kernel: transport; algorithmic bytes per launch / mean launch time
    peak = None
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak_src = "fallback"
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path)).get("hbm_gbs")
        peak_src = "measured"
    if not peak:
        peak = 6650.0
    mean_launch_ms = tt["kernel_ms"] / max(tt["launches"], 1)
    bytes_per_launch = BYTES_PER_SEGMENT_FP64 * tt["segments"] / max(tt["launches"], 1)
    achieved = bytes_per_launch / (mean_launch_ms / 1000.0) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "transport_traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get("dram_bytes_per_launch_fullsize")

    # end to end through the C ABI with host buffers
    e2e = None
    if args.e2e_steps > 0:
        cen = eng.census()
        n = cen.n
        host = Particles(0)
        pin = {}
        for f in Particles.FIELDS:
            pin[f] = torch.empty(max(n, 1) * 2, dtype=torch.float64, pin_memory=True).numpy()
        pin_cell = torch.empty(max(n, 1) * 2, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        host.n = n
        for f in Particles.FIELDS:
            getattr(pin[f], "__setitem__")(slice(0, n), getattr(cen, f))
            setattr(host, f, pin[f][:n])
        pin_cell[:n] = cen.cell
        host.cell = pin_cell[:n]
        host.id = np.zeros(n, np.uint64)
        tempT = torch.empty(p.ncells, dtype=torch.float64, pin_memory=True).numpy()
        torch.cuda.synchronize()
        barrier(dist, "storm")
        t0 = time.perf_counter()
        e2e_segs, h2d, d2h = 0, 0, 0
        for _ in range(args.e2e_steps):
            eng.set_census(host)
            h2d += host.n * (9 * 8 + 4)
            st = eng.step()
            e2e_segs += st["segments"]
            out = eng.census()            # census back to the host
            d2h += out.n * (9 * 8 + 4)
            T = eng.cells()["temperature"]
            tempT[:] = T
            d2h += p.ncells * 8
            nn = out.n
            if nn > len(pin_cell):
                break
            for f in Particles.FIELDS:
                pin[f][:nn] = getattr(out, f)
                setattr(host, f, pin[f][:nn])
            pin_cell[:nn] = out.cell
            host.cell = pin_cell[:nn]
            host.id = np.zeros(nn, np.uint64)
            host.n = nn
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        wall = reduce(dist, wall, "max", "storm")
        e2e_all = reduce(dist, e2e_segs, "sum", "storm")
        e2e = {"value": e2e_all / wall, "unit": UNIT, "h2d_bytes_per_step": int(h2d / args.e2e_steps),
               "d2h_bytes_per_step": int(d2h / args.e2e_steps), "steps": args.e2e_steps,
               "note": "pageable->pinned staging in numpy; copies inside the timed region"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.n, 1)

    if rank == 0:
        lat = sorted(step_ms)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox streams)",
            "config": workload_config(args.n) | {"parallelism": f"{ws} independent problem(s), one per GPU"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "segments_per_step": segs / args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "kernel": "k_transport",
                         "bytes_per_segment": BYTES_PER_SEGMENT_FP64,
                         "mean_launch_ms": mean_launch_ms, "launches": tt["launches"],
                         "peak_source": peak_src},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": ck, "gpu_launches": launches,
            "transport_share": tt["kernel_ms"] / max(sum(step_ms), 1e-9),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        eng.close()
        dist.destroy_process_group()


# ---------------------------------------------------------------------- reference arm
def run_reference(args, ws, rank, dist):
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    cores = os.cpu_count() or 1
    try:   # each reference process holds ~1.5 GB on the 64^3 sample
        import psutil
        cores = max(1, min(cores, int(psutil.virtual_memory().available / 1.5e9)))
    except ImportError:
        pass
    from oracle import ref
    kind = "reference" if ref.available() else "port"
    # each bench step = one bounded sample per core (3 IMC steps, 2 timed)
    total_steps = args.warmup + args.steps
    res = None
    vals = []
    for s in range(max(1, min(total_steps, 2))):
        res = cpu_baseline(args.n, cores)
        if s >= (1 if total_steps > 1 else 0):
            vals.append(res["value"])
    value = statistics.mean(vals) if vals else res["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded std::mt19937_64 in the reference)",
            "config": workload_config(args.n) | {"parallelism": f"{cores} independent reference processes"},
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
