"""Helpers shared by the tests: golden fixtures and case construction."""
from __future__ import annotations

import glob
import os

import numpy as np

from adaptflood_b200 import forcing as fc
from adaptflood_b200 import scenarios as sc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name: str):
    """Returns (case, forcing, expected) for one fixture."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    free = z["free"]
    case = sc.Case(int(z["nx"]), int(z["ny"]), float(z["dx"]), z["dem"], nodata=float(z["nodata"]),
                   fpn=float(z["fpn"]), depth_thresh=float(z["depth_thresh"]), cfl=float(z["cfl"]),
                   init_tstep=float(z["init_tstep"]), sim_time=float(z["sim_time"]),
                   mass_int=float(z["mass_int"]), west_free=bool(free[0]),
                   east_free=bool(free[1]), north_free=bool(free[2]), south_free=bool(free[3]),
                   name=name)
    if z["h0"].size:
        case.h0 = z["h0"]
    f = fc.Forcing(**{k[2:]: z[k] for k in z.files if k.startswith("f_")})
    if f.n_rain:
        case.rain_times, case.rain_rates = f.rain_times, f.rain_rates
    exp = {k: z[k] for k in ("dt", "t_end", "steps", "H", "Qx", "Qy", "Vx", "Vy", "vol", "area",
                             "ref_free", "ref_pt_idx", "ref_pt_type", "ref_pt_value",
                             "ref_pt_nser")}
    return case, f, exp
