"""FP32-versus-FP64 error report of the fused step on one configuration.

Runs the same case with FP64 state (the plain form) and with FP32 state (FP64
time, dt inputs, hydrograph interpolation and volume sums), each from its
initial state to the case's sim_time on the device, and reports

* max and RMS depth error of the FP32 run against the FP64 run (m);
* relative mass error: |V32 - V64| / V64 of the end volumes, and the largest
  such error over the mass reports along the run (FP64-accumulated volumes);
* step counts, end times and rates of both runs.

    python -m adaptflood_b200.accuracy --config 3            # 16384^2, 10800 s
    python -m adaptflood_b200.accuracy --config 3 --size 4096 --sim-time 1800

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


def make_case(config: int, size=None, sim_time=None) -> sc.Case:
    if config == 1:
        case = sc.config1()
    elif config == 2:
        case = sc.config2(n=size or 8192)
    elif config == 3:
        n = size or 16384
        case = sc.config3(n=n, block=min(512, n // 8))
    else:
        raise ValueError(f"unknown configuration {config}")
    if sim_time is not None:
        case.sim_time = float(sim_time)
    return case


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


def report(case: sc.Case, device: int = 0) -> dict:
    r64 = run(case, "f64", device)
    r32 = run(case, "f32", device)
    d = r32["H"] - r64["H"]
    valid = case.dem != case.nodata
    err = np.abs(d[valid])
    k = min(len(r32["mass_v"]), len(r64["mass_v"]))
    # mass reports fall at the first step with t >= each report time; the two
    # runs' dt differ slightly, so compare the reports pairwise by index
    rel_series = (np.abs(r32["mass_v"][:k] - r64["mass_v"][:k]) /
                  np.maximum(np.abs(r64["mass_v"][:k]), 1e-300)) if k else np.zeros(1)
    cells = case.cells
    return {
        "case": case.name, "nx": case.nx, "ny": case.ny, "dx": case.dx,
        "sim_time": case.sim_time,
        "max_depth_error_m": float(err.max()) if err.size else 0.0,
        "rms_depth_error_m": float(np.sqrt(np.mean(err ** 2))) if err.size else 0.0,
        "max_depth_m": float(r64["H"].max()),
        "wet_cells_fp64": int(np.count_nonzero(r64["H"] > 0.001)),
        "relative_mass_error_end": abs(r32["vol"] - r64["vol"]) / abs(r64["vol"]),
        "relative_mass_error_max_over_reports": float(rel_series.max()) if k else None,
        "mass_reports_compared": int(k),
        "volume_fp64_m3": r64["vol"], "volume_fp32_m3": r32["vol"],
        "steps": {"f64": r64["steps"], "f32": r32["steps"]},
        "t_end": {"f64": r64["t_end"], "f32": r32["t_end"]},
        "cell_updates_per_s": {"f64": cells * r64["steps"] / r64["seconds"],
                               "f32": cells * r32["steps"] / r32["seconds"]},
        "seconds": {"f64": r64["seconds"], "f32": r32["seconds"]},
        "tolerance": {"max_depth_error_m": 1e-3, "relative_mass_error": 1e-6},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--sim-time", type=float, default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    case = make_case(a.config, a.size, a.sim_time)
    print(json.dumps(report(case, a.device)))


if __name__ == "__main__":
    main()
