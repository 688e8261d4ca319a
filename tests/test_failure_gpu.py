"""Failure paths of the fused step, made without a GPU fault.

* A diverged state (host-made bad input: an infinite start depth, or a NaN
  CFL number) gives a non-positive or non-finite dt; the step loop stops
  after that step and the call returns AF_ESTATE.  In a batch only that
  member stops (its state reads -1) while the others finish with the same
  results as alone.  Later simulations in the same process run normally.
* A ring wait that runs out: a test build of the library whose ring waits
  give up at once (AF_RING_WAIT_LIMIT=0, built by build.build_wait_test)
  takes the kernels' time-out path -- the warp drains its copies in flight
  (with the normal limit), flags the control block, and the loop stops with
  AF_ESTATE.  It runs in a child process; the same process then still uses
  the device (a fill and a new simulation's creation).
"""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from adaptflood_b200 import _lib
from adaptflood_b200 import build as B
from adaptflood_b200 import forcing as fc
from adaptflood_b200 import scenarios as sc
from adaptflood_b200.batch import Batch
from adaptflood_b200.sim import Simulation
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case(seed=31, nx=90, ny=70):
    c = sc.small_case(nx, ny, seed=seed, sim_time=300.0, n_qfix=1, n_qvar=1, rain=True)
    return c


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("bad", ["inf_depth", "nan_cfl"])
def test_diverged_state_stops_with_estate(cuda, precision, bad):
    case = _case()
    if bad == "inf_depth":
        case.h0 = np.zeros((case.ny, case.nx))
        case.h0[case.ny // 2, case.nx // 3] = np.inf
    else:
        # a wet start, so the first dt already comes from the CFL number (a dry
        # start takes InitTstep, src/kernels.cpp:36-43)
        case.h0 = np.full((case.ny, case.nx), 0.5)
        case.cfl = float("nan")
    f = fc.pack(case)
    with Simulation(case, precision, forcing=f) as s:
        with pytest.raises(_lib.AFError) as e:
            s.run(case.sim_time)
        assert e.value.code == _lib.AF_ESTATE
        t, _, _, steps = s.status()
        # stopped after the step that found dt invalid (dt = 0 or NaN)
        assert steps == 1 and (t == 0.0 if bad == "inf_depth" else np.isnan(t))
        with pytest.raises(_lib.AFError) as e:
            s.run(case.sim_time)  # stays stopped
        assert e.value.code == _lib.AF_ESTATE and s.status()[3] == 1
    # the process and device are still fine: a sound case runs to the oracle's result
    good = _case(seed=32)
    g = fc.pack(good)
    o = orc.OracleSim(good, g)
    n_ref = o.run(good.sim_time)
    with Simulation(good, "f64", forcing=g) as s:
        assert s.run(good.sim_time) == n_ref
        assert np.max(np.abs(s.state()["H"] - o.state(velocity=False)["H"])) <= 1e-9


def test_diverged_member_stops_alone_in_a_batch(cuda):
    bad = _case(seed=33)
    bad.h0 = np.zeros((bad.ny, bad.nx))
    bad.h0[3, 4] = np.inf
    good = _case(seed=34, nx=130, ny=50)
    fb, fg = fc.pack(bad), fc.pack(good)
    with Simulation(good, "f32", forcing=fg) as s:
        n_alone = s.run(good.sim_time)
        h_alone = s.state()["H"]
    with Batch("f32") as b:
        sb = b.add(bad, fb)
        sg = b.add(good, fg)
        b.run()
        t_b, _, _, steps_b, state_b = b.status(sb)
        t_g, _, _, steps_g, state_g = b.status(sg)
        h_g = b.state(sg)["H"]
    assert state_b == -1 and steps_b == 1 and t_b == 0.0
    assert state_g == 1 and steps_g == n_alone and t_g >= good.sim_time
    np.testing.assert_array_equal(h_g, h_alone)


CHILD = textwrap.dedent("""
    import sys
    sys.path.insert(0, {root!r})
    import numpy as np
    import torch
    from adaptflood_b200 import _lib, forcing as fc, scenarios as sc
    from adaptflood_b200.batch import Batch
    from adaptflood_b200.sim import Simulation
    assert _lib.LIB_PATH.endswith("libadaptflood_waittest.so"), _lib.LIB_PATH
    case = sc.small_case(200, 150, seed=41, sim_time=200.0, rain=True)
    f = fc.pack(case)
    out = []
    for prec in ("f64", "f32"):
        with Simulation(case, prec, forcing=f) as s:
            try:
                s.run(case.sim_time)
                out.append("sim-ok")
            except _lib.AFError as e:
                out.append("sim-%d-steps-%d" % (e.code, s.status()[3]))
    with Batch("f32") as b:
        b.add(case, f)
        try:
            b.run()
            out.append("batch-ok")
        except _lib.AFError as e:
            out.append("batch-%d" % e.code)
    # the context is still usable
    x = torch.zeros(1000, dtype=torch.float64, device="cuda")
    import ctypes as C
    rc = _lib.lib().af_fill(C.c_void_p(x.data_ptr()), 1000, 2.5,
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    out.append("fill-%d-%s" % (rc, float(x.sum())))
    with Simulation(case, "f64", forcing=f) as s:
        out.append("create-ok")
    print(" ".join(out))
""")


def test_ring_wait_timeout_reports_estate(cuda):
    B.build_wait_test()  # incremental: rebuilds only what changed since the last build
    env = dict(os.environ, AF_LIB_PATH=B.WAITTEST_LIB)
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    words = r.stdout.split()
    e = _lib.AF_ESTATE
    assert words == [f"sim-{e}-steps-1", f"sim-{e}-steps-1", f"batch-{e}", "fill-0-2500.0",
                     "create-ok"], r.stdout
