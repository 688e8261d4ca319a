"""Python host API over the simulation layer (af_sim_* in include/adaptflood.h).

``Simulation`` owns one device-resident case.  ``run(t_stop)`` is the
reference's time loop ``while (t < sim_time)`` (src/main.cpp:227) as one
CUDA-graph launch; ``state()`` returns full-precision fields in the
reference's layout; ``velocity()`` is ComputeVelocity_GPU
(src/kernels.cpp:293-351) on the device.  ``load_par()`` reads a case from
``.par`` files with the reference's parsing rules.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from . import _lib
from . import forcing as fc
from . import scenarios as sc

_p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731


def case_desc(case: sc.Case) -> _lib.CaseDesc:
    d = _lib.CaseDesc()
    d.nx, d.ny, d.dx, d.nodata = case.nx, case.ny, case.dx, case.nodata
    d.fpn, d.depth_thresh, d.cfl, d.init_tstep = case.fpn, case.depth_thresh, case.cfl, case.init_tstep
    d.g, d.max_hflow, d.theta = 9.81, 10.0, 1.0  # src/main.cpp:118-124
    d.west_free, d.east_free = int(case.west_free), int(case.east_free)
    d.north_free, d.south_free = int(case.north_free), int(case.south_free)
    d.mass_int = case.mass_int
    return d


class _ForcingArrays:
    """Keeps the numpy arrays alive while the C struct points into them."""

    def __init__(self, f: fc.Forcing):
        self.arrays = [np.ascontiguousarray(a) for a in (
            f.flow_idx.astype(np.int32), f.flow_type.astype(np.int32), f.flow_value,
            f.flow_off.astype(np.int32), f.flow_times, f.flow_vals,
            f.other_idx.astype(np.int32), f.other_type.astype(np.int32), f.other_value,
            f.other_off.astype(np.int32), f.other_times, f.other_vals,
            f.rain_times, f.rain_rates)]
        a = self.arrays
        d = _lib.ForcingDesc()
        d.n_flow = f.n_flow
        (d.flow_idx, d.flow_type, d.flow_value, d.flow_off, d.flow_times,
         d.flow_vals) = [x.ctypes.data for x in a[0:6]]
        d.n_other = f.n_other
        (d.other_idx, d.other_type, d.other_value, d.other_off, d.other_times,
         d.other_vals) = [x.ctypes.data for x in a[6:12]]
        d.n_rain = f.n_rain
        d.rain_times, d.rain_rates = a[12].ctypes.data, a[13].ctypes.data
        self.desc = d


class Simulation:
    def __init__(self, case: sc.Case, precision: str = "f64", device: int = 0,
                 forcing: Optional[fc.Forcing] = None):
        self.lib = _lib.lib()
        self.case = case
        self.nx, self.ny = case.nx, case.ny
        self.precision = precision
        prec = {"f64": _lib.AF_PREC_F64, "f32": _lib.AF_PREC_F32}[precision]
        f = _ForcingArrays(forcing if forcing is not None else fc.pack(case))
        dem = np.ascontiguousarray(case.dem, dtype=np.float64)
        h0 = None if case.h0 is None else np.ascontiguousarray(case.h0, dtype=np.float64)
        h = C.c_void_p()
        desc = case_desc(case)
        _lib.check(self.lib.af_sim_create(C.byref(desc), C.byref(f.desc), _p(dem), _p(h0), prec,
                                          device, C.byref(h)), "af_sim_create")
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.af_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------- stepping
    def run(self, t_stop: float, max_steps: int = 10_000_000) -> int:
        n = C.c_int64()
        _lib.check(self.lib.af_sim_run(self.h, float(t_stop), int(max_steps), C.byref(n)),
                   "af_sim_run")
        return n.value

    def launch(self, t_stop: float, max_steps: int = 10_000_000) -> None:
        _lib.check(self.lib.af_sim_launch(self.h, float(t_stop), int(max_steps)), "af_sim_launch")

    def sync(self) -> None:
        _lib.check(self.lib.af_sim_sync(self.h), "af_sim_sync")

    @property
    def stream(self) -> int:
        return self.lib.af_sim_stream(self.h) or 0

    def status(self) -> Tuple[float, float, float, int]:
        t, dt, hm = C.c_double(), C.c_double(), C.c_double()
        n = C.c_int64()
        _lib.check(self.lib.af_sim_status(self.h, C.byref(t), C.byref(dt), C.byref(hm), C.byref(n)),
                   "af_sim_status")
        return t.value, dt.value, hm.value, n.value

    @property
    def t(self) -> float:
        return self.status()[0]

    @property
    def steps(self) -> int:
        return self.status()[3]

    # ---------------------------------------------------------------- state
    def state(self, velocity: bool = False, out: Optional[dict] = None) -> dict:
        """H, Qx, Qy (FP64, reference layout); `out` may supply the arrays
        (e.g. in pinned host memory) as {"H", "Qx", "Qy"} of the right sizes."""
        nx, ny = self.nx, self.ny
        if out is not None:
            H, Qx, Qy = (np.ascontiguousarray(out[k]).reshape(-1) for k in ("H", "Qx", "Qy"))
            assert H.size == nx * ny and Qx.size == Qy.size == (nx + 1) * (ny + 1)
        else:
            H = np.zeros(nx * ny)
            Qx = np.zeros((nx + 1) * (ny + 1))
            Qy = np.zeros((nx + 1) * (ny + 1))
        _lib.check(self.lib.af_sim_get_state(self.h, _p(H), _p(Qx), _p(Qy)), "af_sim_get_state")
        out = {"H": H.reshape(ny, nx), "Qx": Qx.reshape(ny + 1, nx + 1),
               "Qy": Qy.reshape(ny + 1, nx + 1)}
        if velocity:
            out["Vx"], out["Vy"] = self.velocity()
        return out

    def depth(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """H (FP64, reference layout); `out` may supply the array."""
        H = np.zeros(self.nx * self.ny) if out is None else np.ascontiguousarray(out).reshape(-1)
        assert H.size == self.nx * self.ny
        _lib.check(self.lib.af_sim_get_state(self.h, _p(H), None, None), "af_sim_get_state")
        return H.reshape(self.ny, self.nx)

    def set_state(self, H, Qx, Qy, t: float) -> None:
        """Sets the state and time; a field given as None keeps its current value."""
        H, Qx, Qy = (None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                     for a in (H, Qx, Qy))
        _lib.check(self.lib.af_sim_set_state(self.h, _p(H), _p(Qx), _p(Qy), float(t)),
                   "af_sim_set_state")

    def velocity(self):
        Vx = np.zeros(self.nx * self.ny)
        Vy = np.zeros(self.nx * self.ny)
        _lib.check(self.lib.af_sim_velocity(self.h, _p(Vx), _p(Vy)), "af_sim_velocity")
        return Vx.reshape(self.ny, self.nx), Vy.reshape(self.ny, self.nx)

    def volume(self) -> Tuple[float, float]:
        v, a = C.c_double(), C.c_double()
        _lib.check(self.lib.af_sim_volume(self.h, C.byref(v), C.byref(a)), "af_sim_volume")
        return v.value, a.value

    def run_output(self, out_dir: str, sim_time: Optional[float] = None,
                   save_int: Optional[float] = None, voutput: bool = False,
                   async_style: bool = False, stages=None, stage_int: float = 60.0,
                   output_format: int = 0) -> int:
        """Runs to ``sim_time`` writing the reference's files into ``out_dir``
        (af_sim_run_output): H_%04d.asc every ``save_int``, H_final.asc, with
        ``voutput`` the velocity grids, and ``stage.csv`` for ``stages`` (a list
        of (name, i, j) cells); with ``async_style`` and ``output_format`` 1
        (NetCDF) or 2 (both), the saves as records of output.nc.  Returns the
        steps taken."""
        case = self.case
        o = _lib.OutputDesc()
        o.out_dir = os.fsencode(out_dir)
        o.save_int = float(case.save_int if save_int is None else save_int)
        o.voutput, o.async_style = int(voutput), int(async_style)
        o.output_format = int(output_format)
        o.xll, o.yll = case.xll, case.yll
        keep = []
        if stages:
            idx = np.array([j * case.nx + i if 0 <= i < case.nx and 0 <= j < case.ny else -1
                            for _, i, j in stages], dtype=np.int32)
            names = (C.c_char_p * len(stages))(*[n.encode() for n, _, _ in stages])
            keep += [idx, names]
            o.n_stage, o.stage_idx, o.stage_names = len(stages), idx.ctypes.data, C.addressof(names)
            o.stage_int = float(stage_int)
        n = C.c_int64()
        t_end = case.sim_time if sim_time is None else sim_time
        _lib.check(self.lib.af_sim_run_output(self.h, float(t_end), C.byref(o), C.byref(n)),
                   "af_sim_run_output")
        del keep
        return n.value

    def checkpoint(self, path: str) -> None:
        """Writes the whole state to a binary checkpoint (af_sim_checkpoint)."""
        _lib.check(self.lib.af_sim_checkpoint(self.h, os.fsencode(path)), "af_sim_checkpoint")

    def restore(self, path: str) -> None:
        """Loads a checkpoint of the same case and precision (af_sim_restore)."""
        _lib.check(self.lib.af_sim_restore(self.h, os.fsencode(path)), "af_sim_restore")

    def mass_series(self):
        n = C.c_int()
        _lib.check(self.lib.af_sim_mass_series(self.h, None, None, None, 0, C.byref(n)),
                   "af_sim_mass_series")
        k = n.value
        t, v, a = np.zeros(max(k, 1)), np.zeros(max(k, 1)), np.zeros(max(k, 1))
        _lib.check(self.lib.af_sim_mass_series(self.h, _p(t), _p(v), _p(a), k, C.byref(n)),
                   "af_sim_mass_series")
        return t[:k], v[:k], a[:k]


def load_par(path: str) -> Tuple[sc.Case, fc.Forcing]:
    """Parses a ``.par`` case with the library's reader (reference rules)."""
    h = _open_par(path)
    try:
        return _case_of(h, path)
    finally:
        _lib.lib().af_scenario_free(h)


def _open_par(path: str) -> C.c_void_p:
    h = C.c_void_p()
    _lib.check(_lib.lib().af_scenario_load(path.encode(), C.byref(h)), "af_scenario_load " + path)
    return h


def _case_of(h: C.c_void_p, path: str) -> Tuple[sc.Case, fc.Forcing]:
    """The case and forcing of an open scenario (af_scenario_get)."""
    lib = _lib.lib()
    d = _lib.CaseDesc()
    f = _lib.ForcingDesc()
    dem_p = C.POINTER(C.c_double)()
    par = np.zeros(3)
    geo = np.zeros(3)
    _lib.check(lib.af_scenario_get(h, C.byref(d), C.byref(f), C.byref(dem_p), _p(par), _p(geo)),
               "af_scenario_get")
    nx, ny = d.nx, d.ny
    dem = np.ctypeslib.as_array(dem_p, shape=(ny * nx,)).copy().reshape(ny, nx) if nx * ny else \
        np.zeros((ny, nx))

    def arr(ptr, n, dt):
        if n == 0 or not ptr:
            return np.zeros(0, dtype=dt)
        ct = C.c_int if dt == np.int32 else C.c_double
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n,)).copy()

    fo = arr(f.flow_off, f.n_flow + 1, np.int32)
    oo = arr(f.other_off, f.n_other + 1, np.int32)
    forcing = fc.Forcing(
        flow_idx=arr(f.flow_idx, f.n_flow, np.int32), flow_type=arr(f.flow_type, f.n_flow, np.int32),
        flow_value=arr(f.flow_value, f.n_flow, np.float64), flow_off=fo,
        flow_times=arr(f.flow_times, int(fo[-1]) if len(fo) else 0, np.float64),
        flow_vals=arr(f.flow_vals, int(fo[-1]) if len(fo) else 0, np.float64),
        other_idx=arr(f.other_idx, f.n_other, np.int32),
        other_type=arr(f.other_type, f.n_other, np.int32),
        other_value=arr(f.other_value, f.n_other, np.float64), other_off=oo,
        other_times=arr(f.other_times, int(oo[-1]) if len(oo) else 0, np.float64),
        other_vals=arr(f.other_vals, int(oo[-1]) if len(oo) else 0, np.float64),
        rain_times=arr(f.rain_times, f.n_rain, np.float64),
        rain_rates=arr(f.rain_rates, f.n_rain, np.float64))
    case = sc.Case(nx, ny, d.dx, dem, xll=float(geo[0]), yll=float(geo[1]), nodata=d.nodata,
                   sim_time=float(par[0]), save_int=float(par[1]), mass_int=float(par[2]),
                   init_tstep=d.init_tstep, cfl=d.cfl, fpn=d.fpn, depth_thresh=d.depth_thresh,
                   west_free=bool(d.west_free), east_free=bool(d.east_free),
                   north_free=bool(d.north_free), south_free=bool(d.south_free),
                   name=path)
    if forcing.n_rain:
        case.rain_times, case.rain_rates = forcing.rain_times, forcing.rain_rates
    return case, forcing


def par_outputs(path: str) -> dict:
    """The outputs a ``.par`` case asks for, as the reference's CLI reads them
    (af_scenario_output): out_dir, save_int, voutput, async_style,
    output_format, stage_int and the stage points [(name, cell index or -1)]."""
    lib = _lib.lib()
    h = _open_par(path)
    try:
        o = _lib.OutputDesc()
        _lib.check(lib.af_scenario_output(h, C.byref(o)), "af_scenario_output")
        names = C.cast(o.stage_names, C.POINTER(C.c_char_p)) if o.n_stage else None
        idx = C.cast(o.stage_idx, C.POINTER(C.c_int)) if o.n_stage else None
        return {"out_dir": o.out_dir.decode(), "save_int": o.save_int, "voutput": bool(o.voutput),
                "async_style": bool(o.async_style), "output_format": o.output_format,
                "stage_int": o.stage_int,
                "stages": [(names[k].decode(), idx[k]) for k in range(o.n_stage)]}
    finally:
        lib.af_scenario_free(h)


def run_par(path: str, precision: str = "f64", device: int = 0) -> int:
    """Runs a ``.par`` case as the reference's CLI does (src/main.cpp): reads
    its inputs, steps it to sim_time and writes the files it asks for
    (af_sim_run_output with af_scenario_output).  Returns the steps taken."""
    lib = _lib.lib()
    h = _open_par(path)
    try:
        case, forcing = _case_of(h, path)
        o = _lib.OutputDesc()
        _lib.check(lib.af_scenario_output(h, C.byref(o)), "af_scenario_output")
        with Simulation(case, precision, device=device, forcing=forcing) as s:
            n = C.c_int64()
            _lib.check(lib.af_sim_run_output(s.h, float(case.sim_time), C.byref(o), C.byref(n)),
                       "af_sim_run_output")
            return n.value
    finally:
        lib.af_scenario_free(h)
