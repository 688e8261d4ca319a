"""GPU parity of the drop-in layer: each af_* kernel against the oracle's
restatement of the same reference function, on the same inputs.

Tolerances: bit-exact everywhere except the interior face fluxes, whose
pow(hflow, 10/3) comes from CUDA's libm on the GPU and glibc on the CPU
(a few ulp apart); those are held to 1e-13 relative.  The full time loop is
held to the 1e-9 m bar on depth.
"""
import ctypes as C

import numpy as np
import pytest

from _util import golden_names, load_golden
from adaptflood_b200 import _lib
from adaptflood_b200 import kernels as K
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

DEPTH_TOL = 1e-9  # m


def _dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def _host(t):
    return t.cpu().numpy()


def _wet_state(case_name, steps):
    """A realistic mid-run state from the oracle on a golden case."""
    case, f, _ = load_golden(case_name)
    o = orc.OracleSim(case, f)
    o.run(1e30, max_steps=steps)
    st = o.state()
    return case, st


def _ol():
    lib = orc._oracle_lib()
    dp = C.c_void_p
    lib.afo_qx.argtypes = [dp] * 5 + [C.c_int, C.c_int] + [C.c_double] * 8
    lib.afo_qy.argtypes = lib.afo_qx.argtypes
    lib.afo_bcs.argtypes = [dp] * 4 + [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double] + [C.c_int] * 4
    lib.afo_update_h.argtypes = [dp] * 3 + [C.c_int, C.c_int, C.c_double, C.c_double]
    lib.afo_rainfall.argtypes = [dp, dp, C.c_long, C.c_double, C.c_double, C.c_double]
    lib.afo_velocity.argtypes = [dp] * 6 + [C.c_int, C.c_int, C.c_double, C.c_double]
    lib.afo_update_qs.argtypes = [dp] * 4 + [C.c_int, C.c_int, C.c_double]
    lib.afo_find_hmax.argtypes = [dp, dp, C.c_long, C.c_double]
    lib.afo_timestep.argtypes = [C.c_double] * 6
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("name,steps", [("closed_rain_points", 60), ("centre_source", 150),
                                        ("west_north_reservoir", 40), ("narrow_2x9", 20)])
def test_floodplain_q(cuda, name, steps):
    case, st = _wet_state(name, steps)
    nx, ny, dx = case.nx, case.ny, case.dx
    H = st["H"].ravel().copy()
    dem = case.dem.ravel().copy()
    Qxo = st["Qx"].ravel() / dx
    Qyo = st["Qy"].ravel() / dx
    lib = _ol()
    hmax = lib.afo_find_hmax(_p(H), _p(dem), H.size, case.nodata)
    dt = lib.afo_timestep(hmax, case.depth_thresh, case.cfl, dx, 9.81, case.init_tstep)
    Qx = np.full(Qxo.size, 7.0)
    Qy = np.full(Qyo.size, 7.0)
    lib.afo_qx(_p(H), _p(dem), _p(Qx), _p(Qxo), _p(Qyo), nx, ny, dx, case.fpn, case.depth_thresh,
               10.0, dt, 9.81, 1.0, case.nodata)
    lib.afo_qy(_p(H), _p(dem), _p(Qy), _p(Qxo), _p(Qyo), nx, ny, dx, case.fpn, case.depth_thresh,
               10.0, dt, 9.81, 1.0, case.nodata)
    gQx, gQy = _dev(np.full(Qxo.size, 7.0)), _dev(np.full(Qyo.size, 7.0))
    ts = K.FloodplainQ_GPU(_dev(H), _dev(dem), gQx, gQy, _dev(Qxo), _dev(Qyo), nx, ny, dx, dx,
                           case.fpn, case.depth_thresh, 10.0, 0.01, 0.0, 1.0, dx * dx, case.cfl,
                           9.81, case.init_tstep, 1.0, case.nodata)
    assert ts == dt
    for got, want in ((_host(gQx), Qx), (_host(gQy), Qy)):
        # the same expressions and the C library's pow algorithm: bit for bit
        # (untouched entries -- edges, corner slots -- keep their value)
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("free", [(1, 1, 1, 1), (0, 0, 0, 0), (1, 0, 1, 0), (0, 1, 0, 1)])
def test_bcs(cuda, free):
    case, st = _wet_state("closed_rain_points", 80)
    nx, ny, dx = case.nx, case.ny, case.dx
    H = st["H"].ravel().copy()
    H[::7] = 0.0005  # below the 0.001 edge threshold
    dem = case.dem.ravel().copy()
    Qx0 = np.random.default_rng(1).normal(size=(nx + 1) * (ny + 1))
    Qy0 = np.random.default_rng(2).normal(size=(nx + 1) * (ny + 1))
    Qx, Qy = Qx0.copy(), Qy0.copy()
    _ol().afo_bcs(_p(Qx), _p(Qy), _p(H), _p(dem), nx, ny, dx, 9.81, case.nodata, *free)
    gQx, gQy = _dev(Qx0), _dev(Qy0)
    K.BCs_GPU(gQx, gQy, _dev(H), _dev(dem), nx, ny, dx, 9.81, 1.0, case.nodata, *free)
    np.testing.assert_array_equal(_host(gQx), Qx)
    np.testing.assert_array_equal(_host(gQy), Qy)


def test_bcs_rejects_one_column_west_free(cuda):
    import torch
    z = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.AFError) as e:
        K.BCs_GPU(z, z, z, z, 1, 3, 1.0, 9.81, 1.0, -9999.0, 1, 0, 0, 0)
    assert e.value.code == _lib.AF_EINVAL


def test_update_h_rain_qs_velocity(cuda):
    case, st = _wet_state("east_south_rain", 70)
    nx, ny, dx = case.nx, case.ny, case.dx
    lib = _ol()
    H = st["H"].ravel().copy()
    dem = case.dem.ravel().copy()
    Qx = st["Qx"].ravel().copy()
    Qy = st["Qy"].ravel().copy()
    # UpdateH
    Hc = H.copy()
    lib.afo_update_h(_p(Hc), _p(Qx), _p(Qy), nx, ny, dx * dx, 0.731)
    gH = _dev(H)
    K.UpdateH_GPU(gH, _dev(Qx), _dev(Qy), nx, ny, dx * dx, 0.731)
    np.testing.assert_array_equal(_host(gH), Hc)
    # Rainfall (positive, zero and negative rates)
    for rate in (1.3e-5, 0.0, -2e-5):
        Hr = H.copy()
        lib.afo_rainfall(_p(Hr), _p(dem), Hr.size, rate, 0.9, case.nodata)
        g = _dev(H)
        K.Rainfall_GPU(g, _dev(dem), nx, ny, rate, 0.9, case.nodata)
        np.testing.assert_array_equal(_host(g), Hr)
    # UpdateQs
    Qxo, Qyo = np.zeros_like(Qx), np.zeros_like(Qy)
    lib.afo_update_qs(_p(Qx), _p(Qy), _p(Qxo), _p(Qyo), nx, ny, dx)
    gxo, gyo = _dev(np.zeros_like(Qx)), _dev(np.zeros_like(Qy))
    K.UpdateQs_GPU(_dev(Qx), _dev(Qy), gxo, gyo, nx, ny, dx)
    np.testing.assert_array_equal(_host(gxo), Qxo)
    np.testing.assert_array_equal(_host(gyo), Qyo)
    # ComputeVelocity
    Vx, Vy = np.zeros(nx * ny), np.zeros(nx * ny)
    lib.afo_velocity(_p(Vx), _p(Vy), _p(H), _p(dem), _p(Qx), _p(Qy), nx, ny, dx, case.nodata)
    gvx, gvy = _dev(np.ones(nx * ny)), _dev(np.ones(nx * ny))
    K.ComputeVelocity_GPU(gvx, gvy, _dev(H), _dev(dem), _dev(Qx), _dev(Qy), nx, ny, dx, case.nodata)
    np.testing.assert_array_equal(_host(gvx), Vx)
    np.testing.assert_array_equal(_host(gvy), Vy)


@pytest.mark.parametrize("n", [1, 7, 300, 4096, 9000])
def test_point_sources_sorted_scatter(cuda, n):
    import torch
    rng = np.random.default_rng(n)
    ncell = 997
    H = rng.uniform(0, 0.2, ncell)
    idx = rng.integers(0, min(ncell, max(2, n // 3)), n).astype(np.int32)  # many duplicates
    flow = rng.normal(0.0, 0.05, n)
    want = H.copy()
    for k in range(n):  # src/main.cpp:256-260, sequential file order
        want[idx[k]] += flow[k]
        if want[idx[k]] < 0.0:
            want[idx[k]] = 0.0
    g = _dev(H)
    K.AddFlowBCs(g, _dev(idx), _dev(flow), n)
    np.testing.assert_array_equal(_host(g), want)
    # the same with an index off the grid: skipped, and reported
    idx2 = idx.copy()
    idx2[n // 2] = ncell + 5
    g = _dev(H)
    with pytest.raises(_lib.AFError) as e:
        K.AddFlowBCs(g, _dev(idx2), _dev(flow), n)
    assert e.value.code == _lib.AF_ERANGE
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [1, 5, 5000])
def test_apply_point_bcs_last_wins(cuda, n):
    rng = np.random.default_rng(100 + n)
    ncell = 211
    H = rng.uniform(0, 1, ncell)
    idx = rng.integers(0, 50, n).astype(np.int32)
    typ = rng.integers(0, 4, n).astype(np.int32)  # 0 is not a depth BC: no effect
    val = rng.uniform(0, 2, n)
    want = H.copy()
    orc._oracle_lib().afo_point_bcs(_p(want), _p(idx), _p(typ), _p(val), n)
    g = _dev(H)
    K.ApplyPointBCs_GPU(g, _dev(idx), _dev(typ), _dev(val), n, 10, 1.0, 1.0, 1.0)
    np.testing.assert_array_equal(_host(g), want)


def test_volume_area_and_fill(cuda):
    import torch
    rng = np.random.default_rng(5)
    H = rng.uniform(0, 0.05, 1_000_003)
    g = _dev(H)
    v1, a1 = K.VolumeArea(g, 25.0)
    v2, a2 = K.VolumeArea(g, 25.0)
    assert (v1, a1) == (v2, a2)  # fixed summation order
    assert abs(v1 - float(np.sum(H * 25.0))) <= 1e-12 * v1
    assert a1 == float(np.count_nonzero(H > 0.01)) * 25.0
    K.Fill(g, 0.0)
    assert float(torch.count_nonzero(g)) == 0.0
    assert K.VolumeArea(g[:0], 1.0) == (0.0, 0.0)


@pytest.mark.parametrize("name", golden_names())
def test_dropin_loop_matches_reference(cuda, name):
    """The reference's main loop (src/main.cpp:227-288) driven through the
    drop-in kernels only, against the reference's own output."""
    import torch
    case, f, exp = load_golden(name)
    nx, ny, dx = case.nx, case.ny, case.dx
    dA = dx * dx
    F = (nx + 1) * (ny + 1)
    H = _dev(case.h0.ravel() if case.h0 is not None else np.zeros(nx * ny))
    DEM = _dev(case.dem.ravel())
    Qx, Qy, Qxo, Qyo = (torch.zeros(F, dtype=torch.float64, device="cuda") for _ in range(4))
    ps_idx = _dev(f.flow_idx.astype(np.int32))
    bc_idx = _dev(f.other_idx.astype(np.int32))
    bc_type = _dev(f.other_type.astype(np.int32))
    oracle_lib = orc._oracle_lib()
    oracle_lib.afo_interp.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double]

    def interp(times, vals, fixed, t):
        return oracle_lib.afo_interp(_p(times), _p(vals), len(times), fixed, t)

    t, steps = 0.0, 0
    dts = []
    while t < case.sim_time:
        Tstep = K.FloodplainQ_GPU(H, DEM, Qx, Qy, Qxo, Qyo, nx, ny, dx, dx, case.fpn,
                                  case.depth_thresh, 10.0, 0.01, case.init_tstep, 1.0, dA,
                                  case.cfl, 9.81, case.init_tstep, 1.0, case.nodata)
        K.BCs_GPU(Qx, Qy, H, DEM, nx, ny, dx, 9.81, Tstep, case.nodata, case.west_free,
                  case.east_free, case.north_free, case.south_free)
        if f.n_flow:
            flow = np.empty(f.n_flow)
            for k in range(f.n_flow):
                o0, o1 = f.flow_off[k], f.flow_off[k + 1]
                v = f.flow_value[k] if f.flow_type[k] == 4 else interp(
                    f.flow_times[o0:o1].copy(), f.flow_vals[o0:o1].copy(), f.flow_value[k], t)
                flow[k] = v * dx * Tstep / dA
            K.AddFlowBCs(H, ps_idx, _dev(flow), f.n_flow)
        if f.n_rain:
            K.Rainfall_GPU(H, DEM, nx, ny, interp(f.rain_times, f.rain_rates, 0.0, t), Tstep,
                           case.nodata)
        K.UpdateH_GPU(H, Qx, Qy, nx, ny, dA, Tstep)
        if f.n_other:
            val = f.other_value.copy()
            for b in range(f.n_other):
                if f.other_type[b] == 3:
                    o0, o1 = f.other_off[b], f.other_off[b + 1]
                    val[b] = interp(f.other_times[o0:o1].copy(), f.other_vals[o0:o1].copy(),
                                    f.other_value[b], t)
            K.ApplyPointBCs_GPU(H, bc_idx, bc_type, _dev(val), f.n_other, nx, dx, dA, Tstep)
        K.UpdateQs_GPU(Qx, Qy, Qxo, Qyo, nx, ny, dx)
        t += Tstep
        steps += 1
        dts.append(Tstep)
    assert steps == int(exp["steps"])
    np.testing.assert_array_equal(dts, exp["dt"])
    assert np.max(np.abs(_host(H) - exp["H"].ravel())) <= DEPTH_TOL
    Vx = torch.zeros(nx * ny, dtype=torch.float64, device="cuda")
    Vy = torch.zeros_like(Vx)
    K.ComputeVelocity_GPU(Vx, Vy, H, DEM, Qx, Qy, nx, ny, dx, case.nodata)
    assert np.max(np.abs(_host(Vx) - exp["Vx"].ravel())) <= DEPTH_TOL
    assert np.max(np.abs(_host(Vy) - exp["Vy"].ravel())) <= DEPTH_TOL
