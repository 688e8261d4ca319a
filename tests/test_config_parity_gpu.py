"""FP64 parity at the benchmark configurations, against the reference's own
code (``oracle/_ref``, the reference's src/kernels.cpp + the loop of
src/main.cpp:227-304 compiled here; the C restatement where that library is
absent).

* C1, the plain FP64 configuration (512 x 512 at 10 m, a 20 m^3/s QFIX source
  at the centre, FREE edges), run from t = 0 to its sim_time of 3600 s: step
  count, end time, H, Vx, Vy and the volume series at every mass report.
* C2, the large plain run (8192 x 8192 at 5 m, 4096 QVAR hydrographs, rain,
  an HVAR edge depth), the first steps from the flooded start state the
  benchmark times (t = 1800 s, every face wet): dt series, H, Qx, Qy, Vx, Vy.

Tolerances: depth within 1e-9 m and velocity within 1e-9 m/s of the
reference; step counts and dt series equal.
"""
import numpy as np
import pytest

from adaptflood_b200 import forcing as fc
from adaptflood_b200 import scenarios as sc
from adaptflood_b200.sim import Simulation
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

DEPTH_TOL = 1e-9
VEL_TOL = 1e-9
C2_STEPS = 30
C2_START = 1800.0


def _reference(case, forcing):
    if orc.ref_available():
        return orc.RefSim.from_case(case, forcing)
    return orc.OracleSim(case, forcing)


def _max_err(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def test_c1_full_run_matches_reference(cuda):
    case = sc.config1()
    f = fc.pack(case)
    ref = _reference(case, f)
    # src/main.cpp:291-304: volume and flooded area at every mass report.
    want = []
    next_mass = case.mass_int
    dts = []
    while ref.t < case.sim_time:
        t_before = ref.t
        ref.run(1e30, max_steps=1)
        dts.append(ref.t - t_before)
        if ref.t >= next_mass:
            H = ref.state(velocity=False)["H"]
            want.append((ref.t, float(np.sum(H) * case.dx * case.dx)))
            next_mass += case.mass_int
    exp = ref.state(velocity=True)
    with Simulation(case, "f64", forcing=f) as s:
        n = s.run(case.sim_time)
        t, _, _, steps = s.status()
        st = s.state(velocity=True)
        mt, mv, _ = s.mass_series()
    errs = {k: _max_err(st[k], exp[k]) for k in ("H", "Vx", "Vy")}
    print(f"C1 {n} steps, t_end {t:.9f}; max |diff| H {errs['H']:.3e} m, "
          f"Vx {errs['Vx']:.3e}, Vy {errs['Vy']:.3e} m/s")
    assert n == len(dts) == steps
    assert abs(t - ref.t) <= 1e-12 * t
    assert errs["H"] <= DEPTH_TOL
    assert errs["Vx"] <= VEL_TOL
    assert errs["Vy"] <= VEL_TOL
    assert len(mt) == len(want) > 0
    for k, (tw, vw) in enumerate(want):
        assert abs(mt[k] - tw) <= 1e-12 * tw
        assert abs(mv[k] - vw) <= 1e-9 * max(vw, 1.0)


def test_c2_first_steps_match_reference(cuda):
    case = sc.config2()
    h0 = sc.wet_start(case)
    f = fc.pack(case)
    F = (case.nx + 1) * (case.ny + 1)
    zero = np.zeros(F)
    ref = _reference(case, f)
    ref.set_state(h0.ravel(), zero, zero, C2_START)
    ref_dt = ref.run(1e30, max_steps=C2_STEPS, record_dt=True)
    exp = ref.state(velocity=True)
    t_ref = ref.t
    ref.close()
    with Simulation(case, "f64", forcing=f) as s:
        s.set_state(h0, zero, zero, C2_START)
        n = s.run(1e30, max_steps=C2_STEPS)
        t, _, _, _ = s.status()
        st = s.state(velocity=True)
    errs = {k: _max_err(st[k], exp[k]) for k in ("H", "Qx", "Qy", "Vx", "Vy")}
    print(f"C2 {n} steps from t={C2_START}: t_end {t:.9f} (ref {t_ref:.9f}); " +
          ", ".join(f"{k} {v:.3e}" for k, v in errs.items()))
    assert n == len(ref_dt) == C2_STEPS
    assert abs(t - t_ref) <= 1e-12 * t
    assert errs["H"] <= DEPTH_TOL
    scale = max(1.0, float(np.max(np.abs(exp["Qx"]))), float(np.max(np.abs(exp["Qy"]))))
    assert errs["Qx"] <= 1e-9 * scale
    assert errs["Qy"] <= 1e-9 * scale
    assert errs["Vx"] <= VEL_TOL
    assert errs["Vy"] <= VEL_TOL
