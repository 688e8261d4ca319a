"""Throughput benchmark of the local-inertial time step (cell-updates/s).

Headline workload (the large single plain run): an 8192 x 8192 grid at 5 m
with the seeded DEM generator, 4096 QVAR triangular hydrographs at wet-prone
cells, piecewise 0-50 mm/h rain, an HVAR sinusoidal edge depth and FREE
edges, started at t = 1800 s from a flooded state (a 25 mm film on every cell
and the channel filled to 2 m) so that every face is wet.  A step is one time
step of the whole grid: fluxes, edges, sources, rain, depth update, point BCs
and the Hmax reduction that sets the next dt.

Our arm times K steps of the fused kernel (one CUDA-graph launch, CUDA events
on the simulation's stream) in FP32 (the headline `value`) and FP64, reports
the HBM roofline of the step kernel, the end-to-end rate through the public
C ABI with host buffers (median of nine runs, each reported), and the
reference's own CPU code timed on a bounded
sample of the same workload.  Two more legs (N = 1 only):

* `ensemble`: 256 scenarios of 256^2..2048^2 cells, each with its own dt,
  from t = 0 to 1800 s in one batch (FP32 state, FP64 time and mass), timed
  as one run; beside it a sample of the same scenarios on the plain FP64
  single-grid path, one at a time;
* `serving`: Poisson request streams (grids 128^2..4096^2, sim_time
  600..3600 s) served by continuous batching at several rates, p50/p99
  latency from arrival to the depth field on the host, and the same stream
  served one request at a time by the plain FP64 path.

`--impl reference` runs the reference's CPU code alone (oracle/_ref, built
from the reference sources against the Kokkos-API shim), on this host's cores.

N > 1 (torchrun): every rank runs an independent replica of the headline
workload (scaling "weak"; the time step needs no data exchange between
replicas).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from adaptflood_b200 import forcing as fc  # noqa: E402
from adaptflood_b200 import scenarios as sc  # noqa: E402

BYTES_PER_CELL = {"f32": 28, "f64": 56}  # read H, DEM, Qx, Qy; write H', Qx', Qy'
T_START = 1800.0
E2E_TRIALS = 9
STEPS_PER_ITERATION = 4  # step kernels per iteration of the simulation's graph loop


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", choices=["f32", "f64", "batch"], default=None,
                    help="profiling runs: one precision of the single-grid step, or the "
                         "batch step on --batch-copies copies of the --size grid (FP32)")
    ap.add_argument("--batch-copies", type=int, default=16)
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--ensemble", type=int, default=256,
                    help="scenarios of the batched-ensemble leg (0 = skip)")
    ap.add_argument("--serve-requests", type=int, default=32,
                    help="requests per rate of the serving leg (0 = skip)")
    ap.add_argument("--serve-rates", default="10,50,500",
                    help="Poisson arrival rates (req/s) of the serving leg")
    ap.add_argument("--fp64-sample", type=int, default=12,
                    help="ensemble scenarios run one at a time on the plain FP64 path")
    ap.add_argument("--table", action="store_true",
                    help="measure every configuration (C1-C5: GPU FP32 and FP64, the "
                         "reference's CPU code) and print one JSON object instead of the "
                         "benchmark line")
    ap.add_argument("--largest", type=int, default=16384,
                    help="grid size of the largest-configuration leg (C3; 0 = skip)")
    ap.add_argument("--largest-steps", type=int, default=40,
                    help="timed steps of each precision in the largest-configuration leg")
    return ap.parse_args()


def workload(size: int):
    case = sc.config2(n=size)
    case.h0 = sc.wet_start(case)
    return case, fc.pack(case)


def describe(size: int):
    return {"workload": f"C2 large plain run {size}x{size} dx=5m, 4096 QVAR sources, rain, "
                        f"HVAR edge, FREE N/S/E; flooded start at t={T_START:.0f}s",
            "cells": size * size, "start_t_s": T_START,
            "l2": "inputs larger than L2 (state >= 1.9 GB vs 126 MB L2)",
            "parallelism": "replicas"}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # raw samples (the summary goes into the JSON line); BENCH_CLOCKS_DIR
        # keeps them somewhere of the caller's choosing
        d = os.environ.get("BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(d, f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait()
            self.fh.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    pass
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k in range(4) if r[k] == "Active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(rows)}


def cpu_reference(case, forcing, h0, seconds: float, max_steps: int, start: float = T_START,
                  warmup: int = 1):
    """The reference's own code (oracle/_ref) on this host's cores: as many
    steps of the same workload as fit in `seconds` (after `warmup` untimed
    steps)."""
    from oracle import oracle as orc
    if not orc.ref_available():
        return None
    r = orc.RefSim.from_case(case, forcing)
    if start != 0.0:
        F = (case.nx + 1) * (case.ny + 1)
        z = np.zeros(F)
        r.set_state(h0.ravel(), z, z, start)
    r.run(1e30, max_steps=max(1, warmup))
    n = 0
    t0 = time.perf_counter()
    while n < max_steps:
        r.run(1e30, max_steps=1)
        n += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    r.close()
    return {"value": case.cells * n / el, "unit": "cell-updates/s",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
            "kind": "reference", "steps": n, "seconds": el,
            "sample": f"{n} steps of the same {case.nx}x{case.ny} workload from the same start "
                      f"state at t={start:g}s (after {max(1, warmup)} warm-up steps), reference "
                      f"src/kernels.cpp "
                      f"+ main.cpp loop "
                      f"compiled -O3 -fopenmp against the Kokkos-API shim"}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    case, forcing = workload(args.size)
    res = cpu_reference(case, forcing, case.h0, seconds=max(30.0, args.cpu_seconds),
                        max_steps=max(1, args.steps), warmup=args.warmup)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built here"}))
        return
    ms = res["seconds"] * 1e3 / res["steps"]
    print(json.dumps({
        "impl": "reference", "metric": "cell-updates/s", "value": res["value"],
        "unit": "cell-updates/s", "n_gpus": 0, "steps": res["steps"], "warmup": max(1, args.warmup),
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": describe(args.size),
        "cpu_baseline": {"value": res["value"], "unit": "cell-updates/s", "cores": res["cores"],
                         "kind": "reference", "sample": res["sample"]},
        "e2e": {"value": res["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def time_fused(case, forcing, precision, steps, warmup, device, dist=None, start=T_START):
    """K fused steps as one graph launch, CUDA events on the sim's stream."""
    import torch
    from adaptflood_b200.sim import Simulation
    s = Simulation(case, precision, device=device, forcing=forcing)
    if start != 0.0:
        F = (case.nx + 1) * (case.ny + 1)
        zero = np.zeros(F)
        s.set_state(case.h0, zero, zero, start)
    s.run(1e30, max_steps=warmup)
    stream = torch.cuda.ExternalStream(s.stream, device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    e0.record(stream)
    s.launch(1e30, steps)
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1)
    t, dt, hmax, n = s.status()
    s.close()
    return ms, {"t_end": t, "dt_last": dt, "hmax": hmax}


def time_batch_copies(case, forcing, copies, steps, warmup, device):
    """K batch steps of `copies` copies of the flooded workload grid (FP32,
    fixed strip height), CUDA events on the batch's stream."""
    import torch
    from adaptflood_b200.batch import Batch
    with Batch("f32", device=device) as b:
        b.set_balance(0)
        for _ in range(copies):
            b.add(case, forcing, t_stop=1e30)
        b.run(max_steps=warmup)
        stream, e0, e1 = _event_timer(b.stream, device)
        torch.cuda.synchronize(device)
        e0.record(stream)
        b.launch(max_steps=steps)
        e1.record(stream)
        b.sync()
        return e0.elapsed_time(e1), case.cells * copies


def _pinned(a):
    """A copy of `a` in pinned (page-locked) host memory."""
    import torch
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out


def time_e2e(case, forcing, precision, steps, device):
    """The public C ABI end to end with host buffers in pinned memory, all
    inside the timed region: af_sim_create from host arrays (DEM, start depth
    and forcing: H2D), af_sim_set_state for the start time (the fluxes start at
    zero, as after creation), the K steps, and af_sim_get_state of the depth
    field (D2H).  The inputs are in pinned host memory before the timed region."""
    import copy
    import torch
    from adaptflood_b200.sim import Simulation
    c = copy.copy(case)
    c.dem = _pinned(case.dem)
    c.h0 = _pinned(case.h0)
    out = _pinned(np.zeros(case.cells))
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    s = Simulation(c, precision, device=device, forcing=forcing)
    t1 = time.perf_counter()
    s.set_state(None, None, None, T_START)
    t2 = time.perf_counter()
    s.run(1e30, max_steps=steps)
    t3 = time.perf_counter()
    H = s.depth(out=out)
    t4 = time.perf_counter()
    el = t4 - t0
    s.close()
    h2d = c.dem.nbytes + c.h0.nbytes + sum(a.nbytes for a in forcing.__dict__.values())
    phases = {"create_s": t1 - t0, "set_time_s": t2 - t1, "steps_s": t3 - t2,
              "readback_s": t4 - t3}
    return case.cells * steps / el, h2d // steps, H.nbytes // steps, phases


def _event_timer(stream_ptr, device):
    import torch
    stream = torch.cuda.ExternalStream(stream_ptr, device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    return stream, e0, e1


def run_ensemble(args, device, peak):
    """C4: the ensemble in one batch (FP32 state, FP64 time/mass), every
    scenario from t = 0 to its sim_time, one timed launch of the batch loop;
    beside it a sample of the same scenarios on the plain FP64 single-grid
    path, one at a time."""
    import torch
    from adaptflood_b200.batch import Batch, size_class, trace_summary
    from adaptflood_b200.sim import Simulation
    from adaptflood_b200.tune import tune_rows
    cases = sc.config4(count=args.ensemble)
    forcings = [fc.pack(c) for c in cases]
    classes = sorted({size_class(c.nx, c.ny) for c in cases})
    t0 = time.perf_counter()
    rows = tune_rows(classes, "f32", device=device)
    tune_s = time.perf_counter() - t0
    with Batch("f32", device=device, rows=rows) as b:
        need = sum(b.footprint(c, f) for c, f in zip(cases, forcings))
        slots = [b.add(c, f) for c, f in zip(cases, forcings)]
        b.set_trace(1 << 17)
        stream, e0, e1 = _event_timer(b.stream, device)
        torch.cuda.synchronize(device)
        e0.record(stream)
        b.launch()
        e1.record(stream)
        b.sync()
        ms = e0.elapsed_time(e1)
        steps = [b.status(s)[3] for s in slots]
        batch_steps = b.info()["batch_steps"]
        trace = b.trace()
    cu = sum(c.cells * n for c, n in zip(cases, steps))
    value = cu / (ms / 1e3)
    ach = BYTES_PER_CELL["f32"] * value / 1e9
    # plain FP64 path on a sample spread over the size range
    order = sorted(range(len(cases)), key=lambda k: cases[k].cells)
    pick = [order[int(round(q * (len(order) - 1) / max(1, args.fp64_sample - 1)))]
            for q in range(min(args.fp64_sample, len(order)))]
    cu64 = 0
    ms64 = 0.0
    for k in pick:
        with Simulation(cases[k], "f64", device=device, forcing=forcings[k]) as s:
            st, a0, a1 = _event_timer(s.stream, device)
            torch.cuda.synchronize(device)
            a0.record(st)
            s.launch(cases[k].sim_time)
            a1.record(st)
            s.sync()
            ms64 += a0.elapsed_time(a1)
            cu64 += cases[k].cells * s.steps
    v64 = cu64 / (ms64 / 1e3)
    return {
        "workload": f"C4 ensemble: {len(cases)} scenarios, grids log-uniform 256^2..2048^2 "
                    f"(aspect 1:1..1:4, dx 2/5/10 m), n U(0.02,0.08), 1-64 QFIX/QVAR, all "
                    f"edges FREE, each from t=0 to sim_time 1800 s in one batch",
        "cells": sum(c.cells for c in cases), "cell_updates": cu, "batch_steps": batch_steps,
        "scenario_steps": [min(steps), int(np.median(steps)), max(steps)],
        "seconds": ms / 1e3, "value": value, "unit": "cell-updates/s",
        "scenarios_per_s": len(cases) / (ms / 1e3), "dtype": "f32",
        "arena_bytes_used": need,
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "algorithmic_bytes_per_cell": BYTES_PER_CELL["f32"],
                     "note": "whole batch loop (graph launch incl. begin kernel and the tail "
                             "where few scenarios remain) / wall time on the device"},
        "trace": trace_summary(trace, BYTES_PER_CELL["f32"], peak),
        "tuned_rows": {str(k): v for k, v in rows.items()}, "tune_seconds": tune_s,
        "plain_fp64": {"value": v64, "unit": "cell-updates/s", "scenarios": len(pick),
                       "path": "Simulation f64, one scenario at a time, CUDA events around "
                               "each run"},
        "batched_fp32_over_plain_fp64": value / v64,
    }


def run_serving(args, device):
    """C5: Poisson request streams served by continuous batching (FP32, FP64
    accumulators), latency from arrival to the depth field on the host;
    beside it the plain FP64 path serving the same stream one at a time."""
    from adaptflood_b200.batch import size_class
    from adaptflood_b200.serve import Request, Server, poisson_arrivals, serve_one_at_a_time
    from adaptflood_b200.serve import summary
    from adaptflood_b200.tune import tune_rows
    cases = sc.config5(count=args.serve_requests)
    forcings = [fc.pack(c) for c in cases]
    rows = tune_rows(sorted({size_class(c.nx, c.ny) for c in cases}), "f32", device=device)
    rates = [float(x) for x in args.serve_rates.split(",") if x]
    out = {"workload": f"C5 served loop: {len(cases)} requests per rate, grids log-uniform "
                       f"128^2..4096^2, sim_time U(600,3600) s, Poisson arrivals",
           "rates": {}}
    for rate in rates:
        rng = np.random.default_rng(int(rate * 1000) + 7)
        arr = poisson_arrivals(rate, len(cases), rng)
        reqs = [Request(k, float(arr[k]), cases[k], forcings[k]) for k in range(len(cases))]
        with Server("f32", device=device, rows=rows, keep_results=False) as srv:
            srv.run(reqs)
            launches = srv.launches
        sm = summary(reqs)
        sm["launches"] = launches
        out["rates"][str(rate)] = sm
    # the plain FP64 path, one request at a time, at the middle rate
    rate = rates[len(rates) // 2]
    rng = np.random.default_rng(int(rate * 1000) + 7)
    arr = poisson_arrivals(rate, len(cases), rng)
    reqs = [Request(k, float(arr[k]), cases[k], forcings[k]) for k in range(len(cases))]
    serve_one_at_a_time(reqs, "f64", device=device, keep_results=False)
    out["plain_fp64_one_at_a_time"] = dict(summary(reqs), rate=rate)
    return out


def run_largest(args, device, peak):
    """C3, the largest single-GPU configuration: 16384^2 at 2 m with Gaussian
    ponds and a 1 m deep 512^2 reservoir, from its own start state (t = 0),
    K steps of the fused step in FP32 and in FP64 (CUDA events on the
    simulation's stream), each with its HBM roofline, and the reference's CPU
    code on a bounded sample of the same steps."""
    n = args.largest
    case = sc.config3(n=n)
    forcing = fc.pack(case)
    out = {"workload": f"C3 mixed-precision stress {n}x{n} dx=2m, Gaussian ponds, 1 m deep "
                       f"512x512 reservoir, from t=0", "cells": case.cells,
           "steps": args.largest_steps}
    for prec in ("f32", "f64"):
        ms, info = time_fused(case, forcing, prec, args.largest_steps, max(3, args.warmup),
                              device, start=0.0)
        v = case.cells * args.largest_steps / (ms / 1e3)
        ach = BYTES_PER_CELL[prec] * v / 1e9
        out[prec] = {"value": v, "unit": "cell-updates/s", "ms_per_step": ms / args.largest_steps,
                     "roofline": {"achieved": ach, "peak": peak, "frac": ach / peak,
                                  "unit": "GB/s",
                                  "algorithmic_bytes_per_cell": BYTES_PER_CELL[prec]},
                     "state_after": info}
    if not args.no_cpu_baseline:
        cpu = cpu_reference(case, forcing, case.h0, args.cpu_seconds / 2, 20, start=0.0)
        if cpu is not None:
            out["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind",
                                                       "sample")}
    return out


def _full_run(case, forcing, precision, device):
    """One whole run on the fused path from t = 0 to sim_time, timed with
    CUDA events on the simulation's stream; (cell-updates/s, steps)."""
    import torch
    from adaptflood_b200.sim import Simulation
    with Simulation(case, precision, device=device, forcing=forcing) as s:
        st, a0, a1 = _event_timer(s.stream, device)
        torch.cuda.synchronize(device)
        a0.record(st)
        s.launch(case.sim_time)
        a1.record(st)
        s.sync()
        ms = a0.elapsed_time(a1)
        n = s.steps
    return case.cells * n / (ms / 1e3), n


def _cpu_full_run(case, forcing):
    """The reference's own code from t = 0 to sim_time on all host cores."""
    from oracle import oracle as orc
    r = orc.RefSim.from_case(case, forcing)
    t0 = time.perf_counter()
    n = r.run(case.sim_time)
    el = time.perf_counter() - t0
    r.close()
    return case.cells * n / el, n, el


def run_table(args):
    """Every configuration, GPU FP32 / FP64 and the reference's CPU code, for
    the result table of the baseline document (one JSON object)."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    peak, peak_kind = measured_peak()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    rows = {"peak_gbs": peak, "peak_source": peak_kind, "cpu_cores": cores}
    # C1: whole runs (L2-resident state: launch- and latency-bound)
    c1 = sc.config1()
    f1 = fc.pack(c1)
    v64, n64 = _full_run(c1, f1, "f64", local)
    v32, n32 = _full_run(c1, f1, "f32", local)
    vc, nc, el = _cpu_full_run(c1, f1)
    rows["C1"] = {"gpu_f64": v64, "gpu_f32": v32, "steps_f64": n64, "steps_f32": n32,
                  "cpu": vc, "cpu_steps": nc, "cpu_seconds": el,
                  "hbm_frac_f32": BYTES_PER_CELL["f32"] * v32 / 1e9 / peak,
                  "hbm_frac_f64": BYTES_PER_CELL["f64"] * v64 / 1e9 / peak}
    # C2: the benchmark's flooded start, K steps; CPU: 200 steps
    case, forcing = workload(8192)
    r = {}
    for prec in ("f32", "f64"):
        ms, _ = time_fused(case, forcing, prec, args.steps, args.warmup, local)
        r["gpu_" + prec] = case.cells * args.steps / (ms / 1e3)
        r["hbm_frac_" + prec] = BYTES_PER_CELL[prec] * r["gpu_" + prec] / 1e9 / peak
    cpu = cpu_reference(case, forcing, case.h0, 1e9, 200)
    r["cpu"], r["cpu_sample"] = cpu["value"], cpu["sample"]
    rows["C2"] = r
    del case, forcing
    # C3: from its own start, K steps; CPU: 100 steps
    args.largest = 16384
    args.largest_steps = max(args.largest_steps, 40)
    args.no_cpu_baseline = True
    big = run_largest(args, local, peak)
    c3, f3 = sc.config3(), None
    f3 = fc.pack(c3)
    cpu = cpu_reference(c3, f3, c3.h0, 1e9, 100, start=0.0)
    rows["C3"] = {"gpu_f32": big["f32"]["value"], "gpu_f64": big["f64"]["value"],
                  "hbm_frac_f32": big["f32"]["roofline"]["frac"],
                  "hbm_frac_f64": big["f64"]["roofline"]["frac"],
                  "cpu": cpu["value"], "cpu_sample": cpu["sample"]}
    del c3, f3
    # C4: the batch, the plain FP64 sample; CPU: 8 scenarios across the size range,
    # 50 steps each from t = 0
    args.ensemble = 256
    ens = run_ensemble(args, local, peak)
    cases = sc.config4()
    order = sorted(range(len(cases)), key=lambda k: cases[k].cells)
    pick = [order[int(round(q * (len(order) - 1) / 7))] for q in range(8)]
    from oracle import oracle as orc
    cu, el = 0, 0.0
    for k in pick:
        ref = orc.RefSim.from_case(cases[k], fc.pack(cases[k]))
        t0 = time.perf_counter()
        n = ref.run(cases[k].sim_time, max_steps=50)
        el += time.perf_counter() - t0
        cu += cases[k].cells * n
        ref.close()
    rows["C4"] = {"gpu_f32_batch": ens["value"], "hbm_frac_f32": ens["roofline"]["frac"],
                  "gpu_f64_plain": ens["plain_fp64"]["value"], "cpu": cu / el,
                  "cpu_sample": "8 scenarios spread over the size range, 50 steps each from "
                                "t=0", "scenarios_per_s": ens["scenarios_per_s"],
                  "trace": ens.get("trace")}
    # C5: serving
    args.serve_requests = max(args.serve_requests, 32)
    rows["C5"] = run_serving(args, local)
    print(json.dumps(rows))


def traffic_per_cell(kernel_key: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        v = d.get(kernel_key)
        return None if v is None else float(v)
    return None


def run_ours(args, rank: int, world: int):
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = dist_mod
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    case, forcing = workload(args.size)
    peak, peak_kind = measured_peak()

    if args.only == "batch":
        ms, cells = time_batch_copies(case, forcing, args.batch_copies, args.steps, args.warmup,
                                      local)
        if rank == 0:
            print(json.dumps({"profiling_run": "batch", "copies": args.batch_copies,
                              "ms_per_step": ms / args.steps,
                              "cell_updates_per_s": cells * args.steps / (ms / 1e3)}))
        return
    if args.only is not None:
        ms, info = time_fused(case, forcing, args.only, args.steps, args.warmup, local, dist)
        if rank == 0:
            print(json.dumps({"profiling_run": args.only, "ms_per_step": ms / args.steps,
                              "cells": case.cells, "state_after": info}))
        return
    with Clocks(local) as clk:
        ms32, info32 = time_fused(case, forcing, "f32", args.steps, args.warmup, local, dist)
    ms64, info64 = time_fused(case, forcing, "f64", args.steps, args.warmup, local, dist)
    if dist is not None:
        t = torch.tensor([ms32, ms64], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms32, ms64 = float(t[0]), float(t[1])
    cells = case.cells
    value = cells * args.steps * world / (ms32 / 1e3)
    value64 = cells * args.steps * world / (ms64 / 1e3)
    step_ms32 = ms32 / args.steps
    step_ms64 = ms64 / args.steps
    ach32 = BYTES_PER_CELL["f32"] * cells / (step_ms32 / 1e3) / 1e9
    ach64 = BYTES_PER_CELL["f64"] * cells / (step_ms64 / 1e3) / 1e9
    tr32 = traffic_per_cell("k_step_f32")
    tr64 = traffic_per_cell("k_step_f64")
    # The median of E2E_TRIALS end-to-end runs: the host side of a shared GPU
    # box (pinned-memory transfers, allocation) now and then stalls one run
    # for hundreds of ms; every trial is reported.
    trials = [] if args.no_e2e else [time_e2e(case, forcing, "f32", args.steps, local)
                                     for _ in range(E2E_TRIALS)]
    if trials:
        e2e_v, h2d, d2h, phases = sorted(trials, key=lambda r: r[0])[len(trials) // 2]
    else:
        e2e_v, h2d, d2h, phases = 0.0, 0, 0, {}
    if dist is not None:
        t = torch.tensor([e2e_v], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        e2e_v = float(t[0]) * world
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference(case, forcing, case.h0, args.cpu_seconds, 10_000)
    ens = serve = big = None
    if world == 1 and args.largest > 0:
        big = run_largest(args, local, peak)
    if world == 1 and args.ensemble > 0:
        ens = run_ensemble(args, local, peak)
    if world == 1 and args.serve_requests > 0:
        serve = run_serving(args, local)
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_ms32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": describe(args.size),
            "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s",
                         "frac": ach32 / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_cell": BYTES_PER_CELL["f32"],
                         "traffic": None if tr32 is None else tr32 * cells,
                         "kernel": "k_step<float> (fused step)",
                         # the same step in FP64 (the plain form, like-for-like with the
                         # FP64 reference arm) on the same workload
                         "fp64": {"value": value64, "ms_per_step": step_ms64,
                                  "achieved": ach64, "frac": ach64 / peak,
                                  "algorithmic_bytes_per_cell": BYTES_PER_CELL["f64"],
                                  "traffic": None if tr64 is None else tr64 * cells,
                                  "kernel": "k_step<double> (fused step)"}},
            "fp64": {"value": value64, "ms_per_step": step_ms64, "dtype": "f64",
                     "roofline": {"achieved": ach64, "peak": peak, "frac": ach64 / peak,
                                  "unit": "GB/s",
                                  "traffic": None if tr64 is None else tr64 * cells},
                     "fp32_over_fp64": value / value64},
            "e2e": {"value": e2e_v, "unit": "cell-updates/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "path": "af_sim_create (DEM, start depth, forcing) from pinned host arrays, "
                            "K steps, af_sim_get_state of the depth field into pinned host memory",
                    "phases": phases,
                    "trials": [t[0] for t in trials],
                    "statistic": f"median of {len(trials)} runs"},
            # the begin kernel, then whole loop iterations of STEPS_PER_ITERATION
            # step kernels (those past the K-th return at once)
            "gpu_launches": -(-args.steps // STEPS_PER_ITERATION) * STEPS_PER_ITERATION + 1,
            "clocks": clk.summary(),
            "state_after": {"f32": info32, "f64": info64},
        }
        if cpu is not None:
            line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        if big is not None:
            line["largest"] = big
            line["roofline"]["largest_config"] = {
                "workload": big["workload"],
                "f32": {"value": big["f32"]["value"], "frac": big["f32"]["roofline"]["frac"]},
                "f64": {"value": big["f64"]["value"], "frac": big["f64"]["roofline"]["frac"]}}
        if ens is not None:
            line["ensemble"] = ens
        if serve is not None:
            line["serving"] = serve
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.table:
        run_table(args)
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
