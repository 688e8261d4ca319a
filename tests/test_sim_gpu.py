"""GPU parity of the fused time step (af_sim_*): whole runs against the
reference's golden outputs and against the oracle on larger cases that cross
many strips, plus the FP32 path against the FP64 oracle.

Tolerances: FP64 depth and velocity within 1e-9 m (m/s) of the reference;
step counts and end times equal.  FP32: max depth error <= 1e-3 m and
relative volume error <= 1e-6 against FP64.
"""
import numpy as np
import pytest

from _util import golden_names, load_golden
from adaptflood_b200 import forcing as fc
from adaptflood_b200 import scenarios as sc
from adaptflood_b200 import _lib
from adaptflood_b200._lib import AFError
from adaptflood_b200.sim import Simulation
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

DEPTH_TOL = 1e-9
VEL_TOL = 1e-9
FP32_DEPTH_TOL = 1e-3
FP32_MASS_TOL = 1e-6


# FP64 takes one of two step kernels, with the face law inline or out of line
# (AF_SIM_FACE_CALL forces one; the default picks by grid size): both are
# held to the same bars.
FACE_CALL = pytest.mark.parametrize("face_call", ["0", "1"])


@FACE_CALL
@pytest.mark.parametrize("name", golden_names())
def test_fused_fp64_matches_reference(cuda, name, face_call, monkeypatch):
    monkeypatch.setenv("AF_SIM_FACE_CALL", face_call)
    case, f, exp = load_golden(name)
    with Simulation(case, "f64", forcing=f) as s:
        n = s.run(case.sim_time)
        t, _, _, steps = s.status()
        st = s.state(velocity=True)
    assert n == int(exp["steps"]) == steps
    assert abs(t - float(exp["t_end"])) <= 1e-9 * t
    assert np.max(np.abs(st["H"] - exp["H"])) <= DEPTH_TOL
    assert np.max(np.abs(st["Vx"] - exp["Vx"])) <= VEL_TOL
    assert np.max(np.abs(st["Vy"] - exp["Vy"])) <= VEL_TOL
    scale = max(1.0, float(np.max(np.abs(exp["Qx"]))), float(np.max(np.abs(exp["Qy"]))))
    assert np.max(np.abs(st["Qx"] - exp["Qx"])) <= 1e-9 * scale
    assert np.max(np.abs(st["Qy"] - exp["Qy"])) <= 1e-9 * scale


def _strip_edge_case(nx, ny, seed, R_edges=(4, 8, 16, 32), **kw):
    """A case with sources and depth BCs placed on strip boundaries (columns
    around multiples of 60 and 120, rows around multiples of the strip height)."""
    c = sc.small_case(nx, ny, seed=seed, sim_time=kw.pop("sim_time", 400.0), n_qfix=0, n_qvar=0,
                      **kw)
    cols = sorted({x for m in (60, 120) for k in range(1, nx // m + 1)
                   for x in (m * k - 1, m * k, m * k + 1) if x < nx} | {0, 1, nx - 1})
    rows = sorted({y for r in R_edges for k in range(1, ny // r + 1)
                   for y in (r * k - 1, r * k) if y < ny} | {0, ny - 1})
    rng = np.random.default_rng(seed)
    for n in range(24):
        i, j = int(rng.choice(cols)), int(rng.choice(rows))
        if n % 3 == 0:
            c.points.append(sc.PointBC(sc.QFIX, i, j, value=float(rng.uniform(0.3, 2.0))))
        elif n % 3 == 1:
            tt, vv = sc.triangular_hydrograph(float(rng.uniform(0.3, 2.0)), 60.0, 20.0)
            c.points.append(sc.PointBC(sc.QVAR, i, j, name=f"e{n}", times=tt, values=vv))
        else:
            c.points.append(sc.PointBC(sc.HFIX if n % 2 else sc.FREE, i, j, value=0.4))
    return c


@pytest.mark.parametrize("nx,ny,seed,kw", [
    (131, 77, 21, dict(rain=True)),
    (250, 203, 22, dict(free=(1, 0, 1, 1), nodata_block=True, n_hvar=2)),
    (61, 300, 23, dict(free=(0, 1, 0, 1), h0=True)),
])
@FACE_CALL
def test_fused_fp64_matches_oracle_across_strips(cuda, nx, ny, seed, kw, face_call, monkeypatch):
    monkeypatch.setenv("AF_SIM_FACE_CALL", face_call)
    case = _strip_edge_case(nx, ny, seed, **kw)
    f = fc.pack(case)
    o = orc.OracleSim(case, f)
    dts = o.run(case.sim_time, record_dt=True)
    ref = o.state(velocity=True)
    with Simulation(case, "f64", forcing=f) as s:
        n = s.run(case.sim_time)
        st = s.state(velocity=True)
    assert n == len(dts)
    assert np.max(np.abs(st["H"] - ref["H"])) <= DEPTH_TOL
    for k in ("Vx", "Vy"):
        assert np.max(np.abs(st[k] - ref[k])) <= VEL_TOL, k


def test_fp64_kernels_agree_on_a_mid_size_grid(cuda, monkeypatch):
    """A grid of 760 x 700 cells, whose default FP64 kernel has the face law
    out of line: 150 steps equal the inline kernel's bit for bit and the
    oracle's within 1e-9 m."""
    case = _strip_edge_case(760, 700, 24, rain=True, n_hvar=1)
    f = fc.pack(case)
    out = {}
    for mode in (None, "0"):
        if mode is None:
            monkeypatch.delenv("AF_SIM_FACE_CALL", raising=False)
        else:
            monkeypatch.setenv("AF_SIM_FACE_CALL", mode)
        with Simulation(case, "f64", forcing=f) as s:
            s.run(1e30, max_steps=150)
            out[mode] = (s.status(), s.state(velocity=True))
    assert out[None][0] == out["0"][0]
    for k in ("H", "Qx", "Qy", "Vx", "Vy"):
        np.testing.assert_array_equal(out[None][1][k], out["0"][1][k], err_msg=k)
    o = orc.OracleSim(case, f)
    o.run(1e30, max_steps=150)
    ref = o.state(velocity=True)
    assert np.max(np.abs(out[None][1]["H"] - ref["H"])) <= DEPTH_TOL
    for k in ("Vx", "Vy"):
        assert np.max(np.abs(out[None][1][k] - ref[k])) <= VEL_TOL, k


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_row_copy_methods_agree(cuda, prec, monkeypatch):
    """The step reads its rows with one tiled copy per row (small and mid-size
    grids) or four bulk copies (large grids; AF_SIM_TMA forces either): the
    same states bit for bit, here on a case with sources and depth BCs on
    strip edges, nodata and a grid width that ends mid-strip."""
    case = _strip_edge_case(250, 203, 25, free=(1, 0, 1, 1), nodata_block=True, n_hvar=2)
    f = fc.pack(case)
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("AF_SIM_TMA", mode)
        with Simulation(case, prec, forcing=f) as s:
            s.run(case.sim_time)
            out[mode] = (s.status(), s.state(velocity=True), s.mass_series())
    assert out["0"][0] == out["1"][0]
    for k in ("H", "Qx", "Qy", "Vx", "Vy"):
        np.testing.assert_array_equal(out["0"][1][k], out["1"][1][k], err_msg=k)
    for a, b in zip(out["0"][2], out["1"][2]):
        np.testing.assert_array_equal(a, b)


def test_run_in_pieces_is_bit_identical(cuda):
    case, f, exp = load_golden("closed_rain_points")
    with Simulation(case, "f64", forcing=f) as a, Simulation(case, "f64", forcing=f) as b:
        a.run(case.sim_time)
        for t_stop in (13.0, 13.0, 77.7, 150.0):
            b.run(t_stop)
        b.run(1e30, max_steps=5)
        b.run(case.sim_time)
        sa, sb = a.state(), b.state()
        assert a.status() == b.status()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k])


def test_state_round_trip_and_resume(cuda):
    case, f, _ = load_golden("west_north_reservoir")
    o = orc.OracleSim(case, f)
    o.run(100.0)
    mid = o.state()
    t_mid = o.t
    o.run(case.sim_time)
    ref = o.state()
    with Simulation(case, "f64", forcing=f) as s:
        s.set_state(mid["H"], mid["Qx"], mid["Qy"], t_mid)
        got = s.state()
        np.testing.assert_array_equal(got["H"], mid["H"])
        np.testing.assert_array_equal(got["Qx"], mid["Qx"])
        np.testing.assert_array_equal(got["Qy"], mid["Qy"])
        s.run(case.sim_time)
        st = s.state()
    assert np.max(np.abs(st["H"] - ref["H"])) <= DEPTH_TOL


def test_mass_series_matches_reference_reports(cuda):
    case, f, exp = load_golden("centre_source")
    o = orc.OracleSim(case, f)
    want = []
    next_mass = case.mass_int
    while o.t < case.sim_time:  # src/main.cpp:291-304
        o.run(1e30, max_steps=1)
        if o.t >= next_mass:
            H = o.state(velocity=False)["H"]
            want.append((o.t, float(np.sum(H) * case.dx * case.dx),
                         float(np.count_nonzero(H > 0.01)) * case.dx * case.dx))
            next_mass += case.mass_int
    with Simulation(case, "f64", forcing=f) as s:
        s.run(case.sim_time)
        t, v, a = s.mass_series()
        vol_now, area_now = s.volume()
    assert len(t) == len(want) > 0
    for k, (tw, vw, aw) in enumerate(want):
        assert abs(t[k] - tw) <= 1e-9 * tw
        assert abs(v[k] - vw) <= 1e-9 * max(vw, 1.0)
        assert a[k] == aw
    assert abs(vol_now - float(exp["vol"])) <= 1e-9 * float(exp["vol"])
    assert area_now == float(exp["area"])


# Golden cases in the well-conditioned regime.  closed_rain_points ponds
# water 0.5 m deep in a 3 m channel of a closed box, where the reference's
# theta = 1 scheme amplifies any perturbation by about 15 % per step (FP64
# against FP64 with the DEM moved by 1e-9 m diverges the same way), so an
# FP32-versus-FP64 comparison there measures that growth, not FP32 error.
@pytest.mark.parametrize("name", ["centre_source", "east_south_rain"])
def test_fp32_within_tolerance_of_fp64(cuda, name):
    case, f, exp = load_golden(name)
    with Simulation(case, "f32", forcing=f) as s:
        s.run(case.sim_time)
        H = s.depth()
        vol32, _ = s.volume()
    err = np.max(np.abs(H - exp["H"]))
    rel_mass = abs(vol32 - float(exp["vol"])) / float(exp["vol"])
    assert err <= FP32_DEPTH_TOL, err
    assert rel_mass <= FP32_MASS_TOL, rel_mass


def test_fp32_larger_case(cuda):
    case = _strip_edge_case(240, 180, 31, rain=True, sim_time=600.0)
    f = fc.pack(case)
    o = orc.OracleSim(case, f)
    o.run(case.sim_time)
    H64 = o.state(velocity=False)["H"]
    vol64 = float(np.sum(H64)) * case.dx * case.dx
    with Simulation(case, "f32", forcing=f) as s:
        s.run(case.sim_time)
        H = s.depth()
        vol32, _ = s.volume()
    assert np.max(np.abs(H - H64)) <= FP32_DEPTH_TOL
    assert abs(vol32 - vol64) / vol64 <= FP32_MASS_TOL


def test_loaded_par_runs_like_generated_case(cuda, tmp_path):
    from adaptflood_b200.sim import load_par
    _, _, exp = load_golden("free_sources")
    # the generator call that produced the "free_sources" fixture
    case = sc.small_case(40, 32, seed=11, sim_time=300.0, n_qfix=1, n_qvar=2)
    par = case.write(str(tmp_path))
    c2, f2 = load_par(par)
    with Simulation(c2, "f64", forcing=f2) as s:
        s.run(c2.sim_time)
        H = s.depth()
    assert np.max(np.abs(H - exp["H"])) <= DEPTH_TOL


@pytest.mark.parametrize("nx,ny,seed,kw", [
    (131, 77, 21, dict(rain=True)),
    (250, 203, 22, dict(free=(1, 0, 1, 1), nodata_block=True, n_hvar=2)),
])
def test_fused_equals_dropin_kernels_bitwise(cuda, nx, ny, seed, kw):
    """Both GPU paths use the same pow (af_pow.cuh), so the fused kernel -- if
    it keeps the reference's operation order everywhere -- must equal the
    drop-in per-function kernels bit for bit, step after step."""
    import torch
    from adaptflood_b200 import kernels as K
    case = _strip_edge_case(nx, ny, seed, sim_time=150.0, **kw)
    f = fc.pack(case)
    dx, dA = case.dx, case.dx * case.dx
    F = (nx + 1) * (ny + 1)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    H = dev(case.h0.ravel() if case.h0 is not None else np.zeros(nx * ny))
    DEM = dev(case.dem.ravel())
    Qx, Qy, Qxo, Qyo = (torch.zeros(F, dtype=torch.float64, device="cuda") for _ in range(4))
    o = orc.OracleSim(case, f)  # host-side interpolation only
    import ctypes as C
    lib = orc._oracle_lib()
    lib.afo_interp.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double]
    interp = lambda tt, vv, fx, t: lib.afo_interp(tt.ctypes.data, vv.ctypes.data, len(tt), fx, t)  # noqa
    del o
    with Simulation(case, "f64", forcing=f) as s:
        t = 0.0
        for step in range(60):
            Tstep = K.FloodplainQ_GPU(H, DEM, Qx, Qy, Qxo, Qyo, nx, ny, dx, dx, case.fpn,
                                      case.depth_thresh, 10.0, 0.01, case.init_tstep, 1.0, dA,
                                      case.cfl, 9.81, case.init_tstep, 1.0, case.nodata)
            K.BCs_GPU(Qx, Qy, H, DEM, nx, ny, dx, 9.81, Tstep, case.nodata, case.west_free,
                      case.east_free, case.north_free, case.south_free)
            if f.n_flow:
                flow = np.empty(f.n_flow)
                for k in range(f.n_flow):
                    a, b = f.flow_off[k], f.flow_off[k + 1]
                    v = f.flow_value[k] if f.flow_type[k] == 4 else interp(
                        f.flow_times[a:b].copy(), f.flow_vals[a:b].copy(), f.flow_value[k], t)
                    flow[k] = v * dx * Tstep / dA
                K.AddFlowBCs(H, dev(f.flow_idx.astype(np.int32)), dev(flow), f.n_flow)
            if f.n_rain:
                K.Rainfall_GPU(H, DEM, nx, ny, interp(f.rain_times, f.rain_rates, 0.0, t), Tstep,
                               case.nodata)
            K.UpdateH_GPU(H, Qx, Qy, nx, ny, dA, Tstep)
            if f.n_other:
                val = f.other_value.copy()
                for b in range(f.n_other):
                    if f.other_type[b] == 3:
                        a0, a1 = f.other_off[b], f.other_off[b + 1]
                        val[b] = interp(f.other_times[a0:a1].copy(), f.other_vals[a0:a1].copy(),
                                        f.other_value[b], t)
                K.ApplyPointBCs_GPU(H, dev(f.other_idx.astype(np.int32)),
                                    dev(f.other_type.astype(np.int32)), dev(val), f.n_other, nx,
                                    dx, dA, Tstep)
            K.UpdateQs_GPU(Qx, Qy, Qxo, Qyo, nx, ny, dx)
            t += Tstep
            s.run(1e30, max_steps=1)
            st = s.state()
            assert s.t == t
            np.testing.assert_array_equal(st["H"].ravel(), H.cpu().numpy(), err_msg=f"step {step}")
            np.testing.assert_array_equal(st["Qx"].ravel(), Qx.cpu().numpy())
            np.testing.assert_array_equal(st["Qy"].ravel(), Qy.cpu().numpy())


def test_fp32_rain_on_deep_water_conserves_mass(cuda):
    """Light rain on deep water in a closed box: each step's rain is a few
    ulps of the FP32 depth, the case where round-to-nearest loses it
    systematically.  The FP32 volume stays within 1e-6 of the FP64 volume and
    of the volume the rain adds."""
    case = sc.small_case(200, 150, seed=41, free=(0, 0, 0, 0), n_qfix=0, n_qvar=0,
                         sim_time=600.0, channel=False)
    case.h0 = np.full((case.ny, case.nx), 2.0)
    case.rain_times = np.array([0.0, 1e4])
    case.rain_rates = np.array([0.5e-3 / 3600.0] * 2)  # 0.5 mm/h
    f = fc.pack(case)
    vols = {}
    for prec in ("f64", "f32"):
        with Simulation(case, prec, forcing=f) as s:
            s.run(case.sim_time)
            vols[prec], _ = s.volume()
            t = s.t
    v0 = 2.0 * case.cells * case.dx ** 2
    added = 0.5e-3 / 3600.0 * t * case.cells * case.dx ** 2
    assert abs(vols["f64"] - (v0 + added)) <= 1e-9 * v0
    assert abs(vols["f32"] - vols["f64"]) <= FP32_MASS_TOL * vols["f64"]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_checkpoint_restart_is_bit_identical(cuda, tmp_path, prec):
    case = sc.small_case(131, 77, seed=61, rain=True, n_hvar=1, n_qvar=2, sim_time=400.0)
    f = fc.pack(case)
    ck = str(tmp_path / "run.ckpt")
    with Simulation(case, prec, forcing=f) as a:
        a.run(150.0)
        a.checkpoint(ck)
        a.run(case.sim_time)
        ref, ref_mass, ref_status = a.state(), a.mass_series(), a.status()
    with Simulation(case, prec, forcing=f) as b:
        b.restore(ck)
        b.run(case.sim_time)
        st, mass, status = b.state(), b.mass_series(), b.status()
    assert status == ref_status
    for k in ("H", "Qx", "Qy"):
        np.testing.assert_array_equal(st[k], ref[k])
    for x, y in zip(mass, ref_mass):
        np.testing.assert_array_equal(x, y)
    other = "f32" if prec == "f64" else "f64"
    with Simulation(case, other, forcing=f) as c:
        with pytest.raises(AFError):
            c.restore(ck)
    small = sc.small_case(40, 30, seed=62, sim_time=100.0)
    with Simulation(small, prec) as d:
        with pytest.raises(AFError):
            d.restore(ck)
        with pytest.raises(AFError):
            d.restore(str(tmp_path / "missing.ckpt"))
    # same grid size, another case: a different DEM, Manning n, or forcing
    import copy
    dem2 = copy.copy(case)
    dem2.dem = case.dem.copy()
    dem2.dem[10, 20] += 0.25
    fpn2 = copy.copy(case)
    fpn2.fpn = case.fpn * 1.5
    for other_case, other_f in ((dem2, f), (fpn2, f), (case, fc.pack(sc.small_case(
            131, 77, seed=63, rain=True, n_hvar=1, n_qvar=2, sim_time=400.0)))):
        with Simulation(other_case, prec, forcing=other_f) as e:
            with pytest.raises(AFError) as err:
                e.restore(ck)
            assert err.value.code == _lib.AF_EINVAL


def test_step_limits_are_exact(cuda):
    """The graph loop runs several steps per iteration; a launch still takes
    exactly the steps asked for, and stops at its time limit mid-iteration."""
    case, f, _ = load_golden("closed_rain_points")
    with Simulation(case, "f32", forcing=f) as s:
        for k, n in enumerate((1, 2, 3, 5, 7)):
            assert s.run(1e30, max_steps=n) == n
        assert s.status()[3] == 18
        t = s.status()[0]
        s.run(t + 1e-9, max_steps=100)  # one step ends the time limit
        assert s.status()[3] == 19


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_large_fields_round_trip_from_pageable_memory(cuda, prec):
    """Fields of several pinned-buffer loads each (40 MB as FP64) go in and
    come back through the library's staged copies unchanged (FP32: rounded
    to float once)."""
    nx, ny = 2500, 2000
    case = sc.small_case(nx, ny, seed=61, sim_time=60.0)
    rng = np.random.default_rng(61)
    H = rng.uniform(0.0, 3.0, (ny, nx))
    Qx = rng.normal(0.0, 1.0, (ny + 1, nx + 1))  # reference layout: (nx+1)*(ny+1) faces
    Qy = rng.normal(0.0, 1.0, (ny + 1, nx + 1))
    with Simulation(case, prec) as s:
        s.set_state(H, Qx, Qy, 12.5)
        st = s.state()
    cast = (lambda a: a) if prec == "f64" else (lambda a: a.astype(np.float32).astype(np.float64))
    np.testing.assert_array_equal(st["H"], cast(H))
    np.testing.assert_array_equal(st["Qx"][:ny, :], cast(Qx[:ny, :]))
    np.testing.assert_array_equal(st["Qy"][:, :nx], cast(Qy[:, :nx]))


@pytest.mark.parametrize("n,sim_time", [(1024, 900.0)])
def test_fp32_bars_on_a_c3_like_grid(cuda, n, sim_time):
    """The mixed-precision stress configuration on a 1024^2 window of its own
    terrain (Gaussian ponds, the 1 m deep 512^2 reservoir in the middle, the
    dam-break fronts spreading from it over 900 s, closed edges as in the
    configuration; later the fronts reflect off the window's walls into a
    regime where the reference scheme itself diverges).  FP32 state against
    the FP64 run of the same inputs (itself pinned to the reference by the
    FP64 parity tests): max depth error <= 1e-3 m and relative mass error
    <= 1e-6, at the end and at every mass report."""
    case = sc.config3_window(n)
    case.sim_time = sim_time
    case.mass_int = 300.0
    f = fc.pack(case)
    out = {}
    for prec in ("f64", "f32"):
        with Simulation(case, prec, forcing=f) as s:
            s.run(case.sim_time)
            out[prec] = (s.depth(), s.volume()[0], s.mass_series()[1])
    H64, v64, m64 = out["f64"]
    H32, v32, m32 = out["f32"]
    err = float(np.max(np.abs(H32 - H64)))
    k = min(len(m32), len(m64))
    rel = np.abs(m32[:k] - m64[:k]) / m64[:k]
    print(f"C3-like {n}^2 {sim_time:.0f}s: max depth error {err:.3e} m, relative mass error "
          f"end {abs(v32 - v64) / v64:.3e}, max over {k} reports {rel.max():.3e}")
    assert err <= FP32_DEPTH_TOL
    assert abs(v32 - v64) / v64 <= FP32_MASS_TOL
    assert rel.max() <= FP32_MASS_TOL
