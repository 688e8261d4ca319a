"""ctypes access to the CPU checkers (test infrastructure only).

* :class:`OracleSim` -- the plain-C restatement ``af_oracle.c``
  (``_build/libaforacle.so``), built on demand with the system gcc.
* :class:`RefSim` -- the reference's own ``src/kernels.cpp``/``src/io.cpp``
  compiled against the Kokkos-API shim (``_ref/libafref.so``).  It can only be
  built where the reference sources are mounted; elsewhere it is used if a
  prebuilt copy travelled with the tree, else :func:`ref_available` is False.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libaforacle.so")
REF_SO = os.path.join(HERE, "_ref", "libafref.so")
REF_CLI = os.path.join(HERE, "_ref", "lisflood_ref")
POW_SO = os.path.join(HERE, "_build", "libpowcheck.so")
_lock = threading.Lock()
_libs = {}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _make(target: str, ref_dir: str = None) -> None:
    cmd = ["make", "-s", "-C", HERE, target]
    if ref_dir:
        cmd.append("REF=" + ref_dir)
    subprocess.run(cmd, check=True)


def reference_dir():
    """The reference checkout named by AF_REFERENCE_DIR, if it exists here."""
    d = os.environ.get("AF_REFERENCE_DIR")
    return d if d and os.path.isdir(d) else None


def _stale(so: str, sources) -> bool:
    if not os.path.exists(so):
        return True
    t = os.path.getmtime(so)
    return any(os.path.exists(s) and os.path.getmtime(s) > t for s in sources)


def build(ref: bool = True, ref_dir: str = None) -> None:
    """Compile the C restatement and, given the reference checkout (`ref_dir`
    or AF_REFERENCE_DIR), the reference library and CLI."""
    _make("oracle")
    d = ref_dir or reference_dir()
    if ref and d and os.path.isdir(d):
        _make("ref", d)


def _oracle_lib():
    with _lock:
        if "oracle" in _libs:
            return _libs["oracle"]
        if _stale(ORACLE_SO, [os.path.join(HERE, "af_oracle.c"), os.path.join(HERE, "af_oracle.h")]):
            _make("oracle")
        lib = C.CDLL(ORACLE_SO)
        lib.afo_find_hmax.restype = C.c_double
        lib.afo_timestep.restype = C.c_double
        lib.afo_interp.restype = C.c_double
        lib.afo_source_depth.restype = C.c_double
        lib.afo_create.restype = C.c_void_p
        lib.afo_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.afo_destroy.argtypes = [C.c_void_p]
        lib.afo_step.restype = C.c_double
        lib.afo_step.argtypes = [C.c_void_p]
        lib.afo_run.restype = C.c_long
        lib.afo_run.argtypes = [C.c_void_p, C.c_double, C.c_long, C.c_void_p]
        lib.afo_time.restype = C.c_double
        lib.afo_time.argtypes = [C.c_void_p]
        lib.afo_steps.restype = C.c_long
        lib.afo_steps.argtypes = [C.c_void_p]
        lib.afo_get.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        lib.afo_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        _libs["oracle"] = lib
        return lib


def pow_check_lib():
    """The C library's pow and the host build of the restated pow
    (``pow_check.cpp``), over arrays."""
    with _lock:
        if "pow" in _libs:
            return _libs["pow"]
        srcs = [os.path.join(HERE, "pow_check.cpp"),
                os.path.join(HERE, "..", "adaptflood_b200", "csrc", "af_pow.cuh"),
                os.path.join(HERE, "..", "adaptflood_b200", "csrc", "af_pow_tables.h")]
        if _stale(POW_SO, srcs):
            _make("_build/libpowcheck.so")
        lib = C.CDLL(POW_SO)
        for fn in (lib.powc_libc, lib.powc_restated):
            fn.restype = None
            fn.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.c_double]
        lib.powc_mismatch.restype = C.c_long
        lib.powc_mismatch.argtypes = [C.c_void_p, C.c_long, C.c_double]
        _libs["pow"] = lib
        return lib


def ref_available() -> bool:
    if os.path.exists(REF_SO):
        return True
    try:
        build(ref=True)
    except Exception:
        return False
    return os.path.exists(REF_SO)


def _ref_lib():
    with _lock:
        if "ref" in _libs:
            return _libs["ref"]
    if not ref_available():
        raise RuntimeError("reference library unavailable: " + REF_SO)
    with _lock:
        lib = C.CDLL(REF_SO)
        lib.afref_open.restype = C.c_void_p
        lib.afref_open.argtypes = [C.c_char_p, C.c_int]
        lib.afref_close.argtypes = [C.c_void_p]
        lib.afref_info.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.afref_points.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        lib.afref_set_h.argtypes = [C.c_void_p, C.c_void_p]
        lib.afref_run.restype = C.c_long
        lib.afref_run.argtypes = [C.c_void_p, C.c_double, C.c_long, C.c_void_p]
        lib.afref_time.restype = C.c_double
        lib.afref_time.argtypes = [C.c_void_p]
        lib.afref_steps.restype = C.c_long
        lib.afref_steps.argtypes = [C.c_void_p]
        lib.afref_get.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        lib.afref_volume.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.afref_create.restype = C.c_void_p
        lib.afref_create.argtypes = ([C.c_int, C.c_int, C.c_double, C.c_double] + [C.c_void_p] * 3
                                     + [C.c_int] + [C.c_void_p] * 6 + [C.c_int] + [C.c_void_p] * 6
                                     + [C.c_int] + [C.c_void_p] * 2)
        lib.afref_set_state.argtypes = [C.c_void_p] * 4 + [C.c_double]
        _libs["ref"] = lib
        return lib


def _run_chunked(fn, h, t_stop, max_steps, record_dt, chunk=4096):
    """Steps until t >= t_stop or max_steps; returns the dt series or the count."""
    if not record_dt:
        return fn(h, t_stop, max_steps, None)
    out = []
    left = max_steps
    while left > 0:
        buf = np.zeros(min(chunk, left))
        n = fn(h, t_stop, buf.size, buf.ctypes.data_as(C.c_void_p))
        out.append(buf[:n])
        left -= n
        if n < buf.size:
            break
    return np.concatenate(out) if out else np.zeros(0)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _CaseStruct(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_double), ("nodata", C.c_double), ("fpn", C.c_double),
        ("depth_thresh", C.c_double), ("cfl", C.c_double), ("init_tstep", C.c_double),
        ("g", C.c_double), ("max_hflow", C.c_double), ("theta", C.c_double),
        ("west_free", C.c_int), ("east_free", C.c_int), ("north_free", C.c_int),
        ("south_free", C.c_int),
        ("n_flow", C.c_int), ("flow_idx", C.c_void_p), ("flow_type", C.c_void_p),
        ("flow_value", C.c_void_p), ("flow_off", C.c_void_p), ("flow_times", C.c_void_p),
        ("flow_vals", C.c_void_p),
        ("n_other", C.c_int), ("other_idx", C.c_void_p), ("other_type", C.c_void_p),
        ("other_value", C.c_void_p), ("other_off", C.c_void_p), ("other_times", C.c_void_p),
        ("other_vals", C.c_void_p),
        ("n_rain", C.c_int), ("rain_times", C.c_void_p), ("rain_rates", C.c_void_p),
    ]


class OracleSim:
    """The C restatement run on a :class:`adaptflood_b200.scenarios.Case`."""

    def __init__(self, case, forcing):
        self.lib = _oracle_lib()
        self.case = case
        f = forcing
        self._keep = [np.ascontiguousarray(a) for a in (
            f.flow_idx, f.flow_type, f.flow_value, f.flow_off, f.flow_times, f.flow_vals,
            f.other_idx, f.other_type, f.other_value, f.other_off, f.other_times, f.other_vals,
            f.rain_times, f.rain_rates)]
        k = self._keep
        s = _CaseStruct()
        s.nx, s.ny = case.nx, case.ny
        s.dx, s.nodata, s.fpn = case.dx, case.nodata, case.fpn
        s.depth_thresh, s.cfl, s.init_tstep = case.depth_thresh, case.cfl, case.init_tstep
        s.g, s.max_hflow, s.theta = 9.81, 10.0, 1.0
        s.west_free, s.east_free = int(case.west_free), int(case.east_free)
        s.north_free, s.south_free = int(case.north_free), int(case.south_free)
        s.n_flow = f.n_flow
        (s.flow_idx, s.flow_type, s.flow_value, s.flow_off, s.flow_times,
         s.flow_vals) = [a.ctypes.data for a in k[0:6]]
        s.n_other = f.n_other
        (s.other_idx, s.other_type, s.other_value, s.other_off, s.other_times,
         s.other_vals) = [a.ctypes.data for a in k[6:12]]
        s.n_rain = f.n_rain
        s.rain_times, s.rain_rates = k[12].ctypes.data, k[13].ctypes.data
        self._s = s
        dem = np.ascontiguousarray(case.dem, dtype=np.float64)
        h0 = None if case.h0 is None else np.ascontiguousarray(case.h0, dtype=np.float64)
        self.h = self.lib.afo_create(C.byref(s), _p(dem), _p(h0))
        if not self.h:
            raise MemoryError("afo_create failed")

    def close(self):
        if self.h:
            self.lib.afo_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def run(self, t_stop: float, max_steps: int = 1 << 62, record_dt: bool = False):
        return _run_chunked(self.lib.afo_run, self.h, t_stop, max_steps, record_dt)

    @property
    def t(self) -> float:
        return self.lib.afo_time(self.h)

    @property
    def steps(self) -> int:
        return self.lib.afo_steps(self.h)

    def state(self, velocity: bool = True):
        nx, ny = self.case.nx, self.case.ny
        H = np.zeros(nx * ny)
        Qx = np.zeros((nx + 1) * (ny + 1))
        Qy = np.zeros((nx + 1) * (ny + 1))
        Vx = np.zeros(nx * ny) if velocity else None
        Vy = np.zeros(nx * ny) if velocity else None
        self.lib.afo_get(self.h, _p(H), _p(Qx), _p(Qy), _p(Vx), _p(Vy))
        out = {"H": H.reshape(ny, nx), "Qx": Qx.reshape(ny + 1, nx + 1),
               "Qy": Qy.reshape(ny + 1, nx + 1)}
        if velocity:
            out["Vx"] = Vx.reshape(ny, nx)
            out["Vy"] = Vy.reshape(ny, nx)
        return out

    def set_state(self, H, Qx, Qy, t: float):
        H = np.ascontiguousarray(H, dtype=np.float64)
        Qx = np.ascontiguousarray(Qx, dtype=np.float64)
        Qy = np.ascontiguousarray(Qy, dtype=np.float64)
        self.lib.afo_set_state(self.h, _p(H), _p(Qx), _p(Qy), float(t))


class RefSim:
    """The reference's own code path, loaded from a ``.par`` file (or, with
    :meth:`from_case`, from in-memory arrays)."""

    def __init__(self, parfile: str = None, quiet: bool = True, _handle=None):
        self.lib = _ref_lib()
        self.h = _handle if _handle else self.lib.afref_open(parfile.encode(), 1 if quiet else 0)
        if not self.h:
            raise RuntimeError("reference failed to load " + str(parfile))
        dims = np.zeros(2, dtype=np.int32)
        geo = np.zeros(4)
        par = np.zeros(8)
        flags = np.zeros(6, dtype=np.int32)
        self.lib.afref_info(self.h, _p(dims), _p(geo), _p(par), _p(flags))
        self.nx, self.ny = int(dims[0]), int(dims[1])
        self.xll, self.yll, self.cellsize, self.nodata = geo.tolist()
        (self.sim_time, self.save_int, self.mass_int, self.init_tstep, self.cfl, self.fpn,
         self.depth_thresh, rain) = par.tolist()
        self.rain_enabled = bool(rain)
        self.free = tuple(bool(x) for x in flags[:4])  # west, east, north, south
        self.n_flow, self.n_other = int(flags[4]), int(flags[5])

    def close(self):
        if self.h:
            self.lib.afref_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def points(self):
        n = self.n_flow + self.n_other
        idx = np.zeros(max(n, 1), dtype=np.int32)
        typ = np.zeros(max(n, 1), dtype=np.int32)
        val = np.zeros(max(n, 1))
        nser = np.zeros(max(n, 1), dtype=np.int32)
        self.lib.afref_points(self.h, _p(idx), _p(typ), _p(val), _p(nser))
        return idx[:n], typ[:n], val[:n], nser[:n]

    @classmethod
    def from_case(cls, case, forcing):
        lib = _ref_lib()
        f = forcing
        keep = [np.ascontiguousarray(a) for a in (
            f.flow_idx.astype(np.int32), f.flow_type.astype(np.int32), f.flow_value,
            f.flow_off.astype(np.int32), f.flow_times, f.flow_vals,
            f.other_idx.astype(np.int32), f.other_type.astype(np.int32), f.other_value,
            f.other_off.astype(np.int32), f.other_times, f.other_vals, f.rain_times, f.rain_rates)]
        params = np.array([case.sim_time, case.cfl, case.fpn, case.depth_thresh, case.init_tstep,
                           case.mass_int])
        flags = np.array([case.west_free, case.east_free, case.north_free, case.south_free],
                         dtype=np.int32)
        dem = np.ascontiguousarray(case.dem, dtype=np.float64)
        h = lib.afref_create(case.nx, case.ny, case.dx, case.nodata, _p(params), _p(flags), _p(dem),
                             f.n_flow, *[_p(a) for a in keep[0:6]], f.n_other,
                             *[_p(a) for a in keep[6:12]], f.n_rain, _p(keep[12]), _p(keep[13]))
        obj = cls(_handle=h)
        if case.h0 is not None:
            obj.set_h(np.ascontiguousarray(case.h0, dtype=np.float64).ravel())
        return obj

    def set_state(self, H, Qx, Qy, t: float):
        H = np.ascontiguousarray(H, dtype=np.float64)
        Qx = np.ascontiguousarray(Qx, dtype=np.float64)
        Qy = np.ascontiguousarray(Qy, dtype=np.float64)
        self.lib.afref_set_state(self.h, _p(H), _p(Qx), _p(Qy), float(t))

    def set_h(self, H0):
        H0 = np.ascontiguousarray(H0, dtype=np.float64)
        self.lib.afref_set_h(self.h, _p(H0))

    def run(self, t_stop: float, max_steps: int = 1 << 62, record_dt: bool = False):
        return _run_chunked(self.lib.afref_run, self.h, t_stop, max_steps, record_dt)

    @property
    def t(self) -> float:
        return self.lib.afref_time(self.h)

    @property
    def steps(self) -> int:
        return self.lib.afref_steps(self.h)

    def state(self, velocity: bool = True):
        nx, ny = self.nx, self.ny
        H = np.zeros(nx * ny)
        Qx = np.zeros((nx + 1) * (ny + 1))
        Qy = np.zeros((nx + 1) * (ny + 1))
        Vx = np.zeros(nx * ny) if velocity else None
        Vy = np.zeros(nx * ny) if velocity else None
        self.lib.afref_get(self.h, _p(H), _p(Qx), _p(Qy), _p(Vx), _p(Vy))
        out = {"H": H.reshape(ny, nx), "Qx": Qx.reshape(ny + 1, nx + 1),
               "Qy": Qy.reshape(ny + 1, nx + 1)}
        if velocity:
            out["Vx"] = Vx.reshape(ny, nx)
            out["Vy"] = Vy.reshape(ny, nx)
        return out

    def volume(self):
        v = np.zeros(1)
        a = np.zeros(1)
        self.lib.afref_volume(self.h, _p(v), _p(a))
        return float(v[0]), float(a[0])
