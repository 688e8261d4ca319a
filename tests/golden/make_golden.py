"""Generates tests/golden/*.npz from the reference's own code.

Each case is a seeded synthetic input written as .par/.dem/.bci/.bdy/rain
files, loaded by the reference's parsers and stepped by the reference's
src/kernels.cpp and the loop of src/main.cpp:227-288, compiled unmodified for
the CPU against the in-repo Kokkos-API shim (oracle/_ref/libafref.so, built by
`make -C oracle ref` where the reference sources are mounted).

Stored per case: the inputs (DEM, initial depth, forcing tables, scalars), the
reference's own parse of the point boundaries, the dt of every step, and the
final H, Qx, Qy, Vx, Vy in full FP64 plus the volume/area report.

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from adaptflood_b200 import forcing as fc  # noqa: E402
from adaptflood_b200 import scenarios as sc  # noqa: E402
from oracle import oracle as orc  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def cases():
    yield "free_sources", sc.small_case(40, 32, seed=11, sim_time=300.0, n_qfix=1, n_qvar=2)
    yield "closed_rain_points", sc.small_case(37, 29, seed=12, free=(0, 0, 0, 0), sim_time=300.0,
                                              rain=True, n_hfix=1, n_hvar=1, n_free_pts=1,
                                              dup_sources=True, nodata_block=True)
    yield "west_north_reservoir", sc.small_case(33, 45, seed=13, free=(1, 0, 1, 0), sim_time=240.0,
                                                n_qfix=0, n_qvar=3, h0=True)
    yield "east_south_rain", sc.small_case(50, 21, seed=14, free=(0, 1, 0, 1), sim_time=300.0,
                                           rain=True, n_qfix=2, n_qvar=0, nodata_block=True)
    c = sc.small_case(64, 48, seed=15, sim_time=600.0, n_qfix=0, n_qvar=0)
    c.points.append(sc.PointBC(sc.QFIX, 32, 24, value=2.0))
    yield "centre_source", c
    yield "narrow_2x9", sc.small_case(2, 9, seed=16, sim_time=120.0, n_qfix=1, n_qvar=0,
                                      channel=False)


def main():
    if not orc.ref_available():
        raise SystemExit("reference library unavailable (make -C oracle ref)")
    for name, case in cases():
        with tempfile.TemporaryDirectory() as d:
            par = case.write(d)
            r = orc.RefSim(par)
            if case.h0 is not None:
                r.set_h(case.h0.ravel())
            dts = r.run(case.sim_time, record_dt=True)
            st = r.state(velocity=True)
            vol, area = r.volume()
            idx, typ, val, nser = r.points()
            f = fc.pack(case)
            np.savez_compressed(
                os.path.join(OUT, name + ".npz"),
                nx=case.nx, ny=case.ny, dx=case.dx, nodata=case.nodata, fpn=case.fpn,
                depth_thresh=case.depth_thresh, cfl=case.cfl, init_tstep=case.init_tstep,
                sim_time=case.sim_time, mass_int=case.mass_int,
                free=np.array([case.west_free, case.east_free, case.north_free, case.south_free]),
                ref_free=np.array(r.free), dem=case.dem,
                h0=case.h0 if case.h0 is not None else np.zeros((0,)),
                **{"f_" + k: getattr(f, k) for k in f.__dataclass_fields__},
                ref_pt_idx=idx, ref_pt_type=typ, ref_pt_value=val, ref_pt_nser=nser,
                dt=dts, t_end=r.t, steps=r.steps, H=st["H"], Qx=st["Qx"], Qy=st["Qy"],
                Vx=st["Vx"], Vy=st["Vy"], vol=vol, area=area)
            print(f"{name}: {case.nx}x{case.ny}, {len(dts)} steps, t={r.t:.3f}, "
                  f"Hmax={st['H'].max():.4f}, vol={vol:.3f}")


if __name__ == "__main__":
    main()
