"""FP32-versus-FP64 error report of the fused step on one configuration.

Runs the same case with FP64 state (the plain form) and with FP32 state (FP64
time, dt inputs, hydrograph interpolation and volume sums), each from its
initial state to the case's sim_time on the device, and reports

* max and RMS depth error of the FP32 run against the FP64 run (m);
* relative mass error: |V32 - V64| / V64 of the end volumes, and the largest
  such error over the mass reports along the run (FP64-accumulated volumes);
* step counts, end times and rates of both runs;
* with --input-rounding, the same errors of a third run: FP64 arithmetic on
  the DEM and start depth rounded to FP32 (the inputs an FP32 state holds),
  against plain FP64 -- how much of the FP32 run's error the rounding of the
  inputs alone accounts for (the conditioning of the case).

--config 4 / --config 5 report per scenario over a sample of the ensemble
(C4, run as one FP32 batch) or of the served requests (C5, served by
continuous batching at --rate req/s): max depth error and relative mass error
of each scenario against its own FP64 single-grid run.

    python -m adaptflood_b200.accuracy --config 3            # 16384^2, 10800 s
    python -m adaptflood_b200.accuracy --config 3 --size 4096 --sim-time 1800  # a window

prints one JSON line.  Configurations: 1 (512^2 C1), 2 (C2 8192^2), 3 (C3
16384^2 with ponds and a 1 m reservoir block).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import forcing as fc
from . import scenarios as sc
from .sim import Simulation


def make_case(config: int, size=None, sim_time=None, free_edges: bool = False) -> sc.Case:
    if config == 1:
        case = sc.config1()
    elif config == 2:
        case = sc.config2(n=size or 8192)
    elif config == 3:
        # reduced sizes are windows of the full configuration's terrain around
        # its reservoir (a smaller generated grid would have 16x steeper
        # terrain, where the reference scheme itself diverges)
        n = size or 16384
        case = sc.config3() if n == 16384 else sc.config3_window(n)
        if free_edges:
            case.west_free = case.east_free = case.north_free = case.south_free = True
    else:
        raise ValueError(f"unknown configuration {config}")
    if sim_time is not None:
        case.sim_time = float(sim_time)
    return case


def rounded_inputs(case: sc.Case) -> sc.Case:
    """The case with its DEM and start depth rounded to FP32 (held as FP64)."""
    import copy
    c = copy.copy(case)
    c.dem = case.dem.astype(np.float32).astype(np.float64)
    if case.h0 is not None:
        c.h0 = case.h0.astype(np.float32).astype(np.float64)
    return c


def run(case: sc.Case, precision: str, device: int = 0):
    import torch
    f = fc.pack(case)
    with Simulation(case, precision, device=device, forcing=f) as s:
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        n = s.run(case.sim_time)
        el = time.perf_counter() - t0
        t, _, _, _ = s.status()
        H = s.depth()
        vol, area = s.volume()
        mt, mv, ma = s.mass_series()
    return {"steps": n, "t_end": t, "seconds": el, "H": H, "vol": vol, "area": area,
            "mass_t": mt, "mass_v": mv}


def compare(case: sc.Case, r: dict, r64: dict) -> dict:
    """Depth and mass errors of run r against the FP64 run r64."""
    valid = case.dem != case.nodata
    err = np.abs((r["H"] - r64["H"])[valid])
    k = min(len(r["mass_v"]), len(r64["mass_v"]))
    # mass reports fall at the first step with t >= each report time; the two
    # runs' dt differ slightly, so compare the reports pairwise by index
    rel_series = (np.abs(r["mass_v"][:k] - r64["mass_v"][:k]) /
                  np.maximum(np.abs(r64["mass_v"][:k]), 1e-300)) if k else np.zeros(1)
    d = np.where(valid, np.abs(r["H"] - r64["H"]), 0.0)
    j, i = np.unravel_index(int(np.argmax(d)), d.shape)
    return {"max_depth_error_m": float(err.max()) if err.size else 0.0,
            "rms_depth_error_m": float(np.sqrt(np.mean(err ** 2))) if err.size else 0.0,
            "cells_over_1mm": int(np.count_nonzero(err > 1e-3)),
            "worst_cell": {"row": int(j), "col": int(i), "depth_fp64": float(r64["H"][j, i]),
                           "depth": float(r["H"][j, i])},
            "relative_mass_error_end": abs(r["vol"] - r64["vol"]) / max(abs(r64["vol"]), 1e-300),
            "relative_mass_error_max_over_reports": float(rel_series.max()) if k else None,
            "mass_reports_compared": int(k)}


def report(case: sc.Case, device: int = 0, input_rounding: bool = False) -> dict:
    r64 = run(case, "f64", device)
    r32 = run(case, "f32", device)
    c32 = compare(case, r32, r64)
    cells = case.cells
    out = {
        "case": case.name, "nx": case.nx, "ny": case.ny, "dx": case.dx,
        "sim_time": case.sim_time,
        **c32,
        "max_depth_m": float(r64["H"].max()),
        "wet_cells_fp64": int(np.count_nonzero(r64["H"] > 0.001)),
        "volume_fp64_m3": r64["vol"], "volume_fp32_m3": r32["vol"],
        "steps": {"f64": r64["steps"], "f32": r32["steps"]},
        "t_end": {"f64": r64["t_end"], "f32": r32["t_end"]},
        "cell_updates_per_s": {"f64": cells * r64["steps"] / r64["seconds"],
                               "f32": cells * r32["steps"] / r32["seconds"]},
        "seconds": {"f64": r64["seconds"], "f32": r32["seconds"]},
        "tolerance": {"max_depth_error_m": 1e-3, "relative_mass_error": 1e-6},
    }
    if input_rounding:
        rr = run(rounded_inputs(case), "f64", device)
        out["fp64_on_fp32_rounded_inputs"] = dict(compare(case, rr, r64), volume_m3=rr["vol"],
                                                  steps=rr["steps"])
    return out


# A scenario is called well-conditioned when FP64 arithmetic on its inputs
# rounded to FP32 stays this close to plain FP64 (a tenth of the FP32 bars).
COND_DEPTH_M, COND_MASS = 1e-4, 1e-7


def _scenario_errors(cases, results32, device):
    """Per scenario: the FP32 result (depth field, end volume) against the
    scenario's own FP64 single-grid run, and the scenario's conditioning: the
    same errors of FP64 on the FP32-rounded DEM (and start depth)."""
    rows = []
    for case, (H32, vol32) in zip(cases, results32):
        r64 = run(case, "f64", device)
        rr = run(rounded_inputs(case), "f64", device)
        valid = case.dem != case.nodata
        err = np.abs((H32 - r64["H"])[valid])
        cerr = np.abs((rr["H"] - r64["H"])[valid])
        v64 = max(abs(r64["vol"]), 1e-300)
        row = {"name": case.name, "cells": case.cells, "dx": case.dx,
               "max_depth_error_m": float(err.max()) if err.size else 0.0,
               "relative_mass_error_end": abs(vol32 - r64["vol"]) / v64,
               "conditioning_depth_m": float(cerr.max()) if cerr.size else 0.0,
               "conditioning_mass": abs(rr["vol"] - r64["vol"]) / v64}
        row["well_conditioned"] = (row["conditioning_depth_m"] <= COND_DEPTH_M and
                                   row["conditioning_mass"] <= COND_MASS)
        rows.append(row)

    def stats(rs):
        if not rs:
            return {"scenarios": 0}
        md = [r["max_depth_error_m"] for r in rs]
        mm = [r["relative_mass_error_end"] for r in rs]
        return {"scenarios": len(rs), "max_depth_error_m": max(md),
                "median_max_depth_error_m": float(np.median(md)),
                "relative_mass_error_max": max(mm),
                "relative_mass_error_median": float(np.median(mm)),
                "within_bars": sum(1 for r in rs if r["max_depth_error_m"] <= 1e-3 and
                                   r["relative_mass_error_end"] <= 1e-6)}
    good = [r for r in rows if r["well_conditioned"]]
    return {**stats(rows), "well_conditioned": stats(good),
            "ill_conditioned": stats([r for r in rows if not r["well_conditioned"]]),
            "conditioning_rule": f"FP64 on FP32-rounded inputs within {COND_DEPTH_M} m and "
                                 f"{COND_MASS} relative mass of plain FP64",
            "per_scenario": rows,
            "tolerance": {"max_depth_error_m": 1e-3, "relative_mass_error": 1e-6}}


def ensemble_report(count: int = 16, device: int = 0) -> dict:
    """C4: a sample spread over the ensemble's size range, run as one FP32
    batch, each member against its FP64 single-grid run."""
    from .batch import Batch
    cases = sc.config4()
    order = sorted(range(len(cases)), key=lambda k: cases[k].cells)
    pick = [cases[order[int(round(q * (len(order) - 1) / max(1, count - 1)))]]
            for q in range(count)]
    with Batch("f32", device=device) as b:
        slots = [b.add(c, fc.pack(c)) for c in pick]
        b.run()
        res = []
        for c, sl in zip(pick, slots):
            H = b.depth(sl)
            res.append((H, float(np.sum(H) * c.dx * c.dx)))
    out = _scenario_errors(pick, res, device)
    out["workload"] = f"C4 sample of {count} scenarios across the size range, one FP32 batch"
    return out


def served_report(count: int = 32, rate: float = 50.0, device: int = 0) -> dict:
    """C5: the served requests (continuous batching at `rate` req/s), each
    result against the request's FP64 single-grid run."""
    from .serve import Request, Server, poisson_arrivals
    cases = sc.config5(count=count)
    rng = np.random.default_rng(int(rate * 1000) + 7)
    arr = poisson_arrivals(rate, len(cases), rng)
    reqs = [Request(k, float(arr[k]), cases[k], fc.pack(cases[k])) for k in range(len(cases))]
    with Server("f32", device=device, keep_results=True) as srv:
        srv.run(reqs)
    res = []
    for c, r in zip(cases, reqs):
        H = r.result
        res.append((H, float(np.sum(H) * c.dx * c.dx)))
    out = _scenario_errors(cases, res, device)
    out["workload"] = f"C5: {count} requests served by continuous batching at {rate} req/s"
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--sim-time", type=float, default=None)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--input-rounding", action="store_true",
                    help="also run FP64 on the FP32-rounded DEM and start depth")
    ap.add_argument("--count", type=int, default=None, help="scenarios (configs 4 and 5)")
    ap.add_argument("--rate", type=float, default=50.0, help="arrival rate (config 5)")
    ap.add_argument("--free-edges", action="store_true",
                    help="free outflow at every edge (config 3 windows)")
    a = ap.parse_args()
    if a.config == 4:
        print(json.dumps(ensemble_report(a.count or 16, a.device)))
    elif a.config == 5:
        print(json.dumps(served_report(a.count or 32, a.rate, a.device)))
    else:
        case = make_case(a.config, a.size, a.sim_time, a.free_edges)
        print(json.dumps(report(case, a.device, a.input_rounding)))


if __name__ == "__main__":
    main()
