"""The reference's kernel interface (src/kernels.hpp:8-37), on device tensors.

Each function has the name, argument order and meaning of its reference
counterpart and calls the drop-in C ABI (af_* in include/adaptflood.h).
Arrays are CUDA float64 tensors (int32 for index/type arrays) in the
reference's layout: cells ``i + j*xsz``, faces ``i + j*(xsz+1)``.  Calls are
synchronous, as the reference's functions end in ``Kokkos::fence()``; errors
raise :class:`adaptflood_b200._lib.AFError` where the reference would abort.
``FloodplainQ_GPU`` returns the new ``Tstep`` (the reference's out-parameter).
"""
from __future__ import annotations

import ctypes as C

from . import _lib


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("device tensor required (no CPU fallback)")
    if not t.is_contiguous():
        raise ValueError("contiguous tensor required")
    return C.c_void_p(t.data_ptr())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def UpdateQs_GPU(Qx, Qy, Qxold, Qyold, xsz, ysz, dx):
    _lib.check(_lib.lib().af_update_qs(_ptr(Qx), _ptr(Qy), _ptr(Qxold), _ptr(Qyold), xsz, ysz,
                                       dx, _stream()), "UpdateQs_GPU")


def FloodplainQ_GPU(H, DEM, Qx, Qy, Qxold, Qyold, xsz, ysz, dx, dy, FPn, DepthThresh, MaxHflow,
                    dhlin, Tstep, Qlimfact, dA, cfl, g, InitTstep, theta, nodata):
    ts = C.c_double(Tstep)
    _lib.check(_lib.lib().af_floodplain_q(
        _ptr(H), _ptr(DEM), _ptr(Qx), _ptr(Qy), _ptr(Qxold), _ptr(Qyold), xsz, ysz, dx, dy, FPn,
        DepthThresh, MaxHflow, dhlin, C.byref(ts), Qlimfact, dA, cfl, g, InitTstep, theta, nodata,
        _stream()), "FloodplainQ_GPU")
    return ts.value


def BCs_GPU(Qx, Qy, H, DEM, xsz, ysz, dx, g, dt, nodata, west_free, east_free, north_free,
            south_free):
    _lib.check(_lib.lib().af_bcs(_ptr(Qx), _ptr(Qy), _ptr(H), _ptr(DEM), xsz, ysz, dx, g, dt,
                                 nodata, int(west_free), int(east_free), int(north_free),
                                 int(south_free), _stream()), "BCs_GPU")


def ApplyPointBCs_GPU(H, bc_idx, bc_type, bc_value, num_bcs, ncols, dx, dA, Tstep):
    _lib.check(_lib.lib().af_apply_point_bcs(_ptr(H), _ptr(bc_idx), _ptr(bc_type), _ptr(bc_value),
                                             num_bcs, ncols, dx, dA, Tstep, H.numel(), _stream()),
               "ApplyPointBCs_GPU")


def UpdateH_GPU(H, Qx, Qy, xsz, ysz, dA, Tstep):
    _lib.check(_lib.lib().af_update_h(_ptr(H), _ptr(Qx), _ptr(Qy), xsz, ysz, dA, Tstep, _stream()),
               "UpdateH_GPU")


def ComputeVelocity_GPU(Vx_out, Vy_out, H, DEM, Qx, Qy, xsz, ysz, dx, nodata):
    _lib.check(_lib.lib().af_compute_velocity(_ptr(Vx_out), _ptr(Vy_out), _ptr(H), _ptr(DEM),
                                              _ptr(Qx), _ptr(Qy), xsz, ysz, dx, nodata, _stream()),
               "ComputeVelocity_GPU")


def Rainfall_GPU(H, DEM, xsz, ysz, rain_rate, Tstep, nodata):
    _lib.check(_lib.lib().af_rainfall(_ptr(H), _ptr(DEM), xsz, ysz, rain_rate, Tstep, nodata,
                                      _stream()), "Rainfall_GPU")


def AddFlowBCs(H, ps_idx, ps_flow, num_flow_bcs):
    """The inline point-source scatter of src/main.cpp:256-260."""
    _lib.check(_lib.lib().af_add_point_sources(_ptr(H), _ptr(ps_idx), _ptr(ps_flow), num_flow_bcs,
                                               H.numel(), _stream()), "AddFlowBCs")


def VolumeArea(H, dA):
    """The inline Vol/Area reductions of src/main.cpp:293-298."""
    v, a = C.c_double(), C.c_double()
    _lib.check(_lib.lib().af_volume_area(_ptr(H), H.numel(), dA, C.byref(v), C.byref(a),
                                         _stream()), "VolumeArea")
    return v.value, a.value


def Fill(x, value):
    """The inline Init* fills of src/main.cpp:156-160."""
    _lib.check(_lib.lib().af_fill(_ptr(x), x.numel(), value, _stream()), "Fill")
