"""ctypes binding of libadaptflood.so (the C ABI declared in include/adaptflood.h).

The library is loaded from this package directory.  There is no fallback: if
the shared library is missing, importing anything that needs it raises, so a
run can never silently compute on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
# AF_LIB_PATH selects another build of the same library (e.g. to compare
# code shapes); by default the in-tree build next to this file is used.
LIB_PATH = os.environ.get("AF_LIB_PATH") or os.path.join(HERE, "libadaptflood.so")

AF_OK, AF_EINVAL, AF_ERANGE, AF_ECUDA, AF_ENOMEM, AF_EIO, AF_ESTATE = 0, -1, -2, -3, -4, -5, -6
AF_PREC_F64, AF_PREC_F32 = 0, 1


class AFError(RuntimeError):
    def __init__(self, code: int, what: str):
        lib = _load()
        msg = lib.af_strerror(code).decode()
        if code == AF_ECUDA:
            msg += " (" + lib.af_last_cuda_error().decode() + ")"
        super().__init__(f"{what}: {msg} [{code}]")
        self.code = code


class CaseDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("nodata", C.c_double),
        ("fpn", C.c_double), ("depth_thresh", C.c_double), ("cfl", C.c_double),
        ("init_tstep", C.c_double), ("g", C.c_double), ("max_hflow", C.c_double),
        ("theta", C.c_double), ("west_free", C.c_int), ("east_free", C.c_int),
        ("north_free", C.c_int), ("south_free", C.c_int), ("mass_int", C.c_double),
    ]


class OutputDesc(C.Structure):
    _fields_ = [
        ("out_dir", C.c_char_p), ("save_int", C.c_double), ("voutput", C.c_int),
        ("async_style", C.c_int), ("xll", C.c_double), ("yll", C.c_double),
        ("n_stage", C.c_int), ("stage_idx", C.c_void_p), ("stage_names", C.c_void_p),
        ("stage_int", C.c_double), ("output_format", C.c_int),
    ]


class ForcingDesc(C.Structure):
    _fields_ = [
        ("n_flow", C.c_int), ("flow_idx", C.c_void_p), ("flow_type", C.c_void_p),
        ("flow_value", C.c_void_p), ("flow_off", C.c_void_p), ("flow_times", C.c_void_p),
        ("flow_vals", C.c_void_p),
        ("n_other", C.c_int), ("other_idx", C.c_void_p), ("other_type", C.c_void_p),
        ("other_value", C.c_void_p), ("other_off", C.c_void_p), ("other_times", C.c_void_p),
        ("other_vals", C.c_void_p),
        ("n_rain", C.c_int), ("rain_times", C.c_void_p), ("rain_rates", C.c_void_p),
    ]


_lock = threading.Lock()
_lib = None

_vp, _i, _d, _i64, _u64 = C.c_void_p, C.c_int, C.c_double, C.c_int64, C.c_uint64
_SIGS = {
    "af_strerror": (C.c_char_p, [_i]),
    "af_last_cuda_error": (C.c_char_p, []),
    "af_version": (_i, []),
    "af_update_qs": (_i, [_vp, _vp, _vp, _vp, _i, _i, _d, _vp]),
    "af_floodplain_q": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _d, _d, _d, _d, _d, _d,
                             _vp, _d, _d, _d, _d, _d, _d, _d, _vp]),
    "af_bcs": (_i, [_vp, _vp, _vp, _vp, _i, _i, _d, _d, _d, _d, _i, _i, _i, _i, _vp]),
    "af_apply_point_bcs": (_i, [_vp, _vp, _vp, _vp, _i, _i, _d, _d, _d, _i, _vp]),
    "af_update_h": (_i, [_vp, _vp, _vp, _i, _i, _d, _d, _vp]),
    "af_compute_velocity": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _d, _d, _vp]),
    "af_rainfall": (_i, [_vp, _vp, _i, _i, _d, _d, _d, _vp]),
    "af_add_point_sources": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "af_add_point_sources_noalloc": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "af_volume_area": (_i, [_vp, _i64, _d, _vp, _vp, _vp]),
    "af_fill": (_i, [_vp, _i64, _d, _vp]),
    "af_pow_eval": (_i, [_vp, _vp, _i64, _d, _vp]),
    "af_sim_create": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "af_sim_destroy": (_i, [_vp]),
    "af_sim_launch": (_i, [_vp, _d, _i64]),
    "af_sim_sync": (_i, [_vp]),
    "af_sim_run": (_i, [_vp, _d, _i64, _vp]),
    "af_sim_status": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "af_sim_stream": (_vp, [_vp]),
    "af_sim_get_state": (_i, [_vp, _vp, _vp, _vp]),
    "af_sim_set_state": (_i, [_vp, _vp, _vp, _vp, _d]),
    "af_sim_velocity": (_i, [_vp, _vp, _vp]),
    "af_sim_volume": (_i, [_vp, _vp, _vp]),
    "af_sim_mass_series": (_i, [_vp, _vp, _vp, _vp, _i, _vp]),
    "af_sim_run_output": (_i, [_vp, _d, _vp, _vp]),
    "af_sim_checkpoint": (_i, [_vp, C.c_char_p]),
    "af_sim_restore": (_i, [_vp, C.c_char_p]),
    "af_write_asc": (_i, [C.c_char_p, _vp, _i, _i, _d, _d, _d, _d, _i]),
    "af_netcdf_create": (_i, [C.c_char_p, _i, _i, _i, _d, _d, _d, _d, _vp]),
    "af_netcdf_append": (_i, [_vp, _d, _vp, _vp, _vp]),
    "af_netcdf_close": (_i, [_vp]),
    "af_batch_create": (_i, [_i, _i, _u64, _i, _vp]),
    "af_batch_destroy": (_i, [_vp]),
    "af_batch_size_class": (_i, [_i, _i]),
    "af_batch_set_rows": (_i, [_vp, _i, _i]),
    "af_batch_get_rows": (_i, [_vp, _i]),
    "af_batch_footprint": (_i, [_vp, _vp, _vp, _d, _vp]),
    "af_batch_add": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _vp]),
    "af_batch_remove": (_i, [_vp, _i]),
    "af_batch_launch": (_i, [_vp, _i64, _i]),
    "af_batch_attention": (_i, [_vp]),
    "af_batch_query": (_i, [_vp]),
    "af_batch_sync": (_i, [_vp]),
    "af_batch_run": (_i, [_vp, _i64, _vp]),
    "af_batch_set_balance": (_i, [_vp, _i]),
    "af_batch_slot_status": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "af_batch_get_state": (_i, [_vp, _i, _vp, _vp, _vp]),
    "af_batch_mass_series": (_i, [_vp, _i, _vp, _vp, _vp, _i, _vp]),
    "af_batch_info": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "af_batch_set_trace": (_i, [_vp, _i64]),
    "af_batch_get_trace": (_i, [_vp, _vp, _i64, _vp]),
    "af_batch_stream": (_vp, [_vp]),
    "af_arena_create": (_i, [_u64, _vp]),
    "af_arena_destroy": (_i, [_vp]),
    "af_arena_alloc": (_i, [_vp, _u64, _vp]),
    "af_arena_free": (_i, [_vp, _u64]),
    "af_arena_stats": (_i, [_vp, _vp, _vp, _vp]),
    "af_scenario_load": (_i, [C.c_char_p, _vp]),
    "af_scenario_free": (None, [_vp]),
    "af_scenario_get": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "af_scenario_output": (_i, [_vp, _vp]),
}


def _load():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python adaptflood_b200/build.py` "
                "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def lib():
    return _load()


def check(code: int, what: str) -> None:
    if code != AF_OK:
        raise AFError(code, what)
