"""Flat forcing tables for one case: point sources, point depth BCs, rain.

The tables mirror what src/main.cpp:77-194 builds from the parsed point
boundaries: flow boundaries (QFIX/QVAR) and "other" boundaries
(FREE/HFIX/HVAR, typed 1/2/3 as on the device, src/main.cpp:187-189), each in
file order, plus the uniform rain series (src/types.hpp:86-90).  Hydrographs
are stored in CSR form: entries ``off[k]..off[k+1]`` of ``times``/``vals``.
A series with no entries interpolates to the fixed value, as
``interpolate_bc_value`` does for a boundary the ``.bdy`` file never named
(src/io.cpp:300).
"""
from __future__ import annotations

import dataclasses
from typing import List

import numpy as np

from . import scenarios as sc


@dataclasses.dataclass
class Forcing:
    flow_idx: np.ndarray
    flow_type: np.ndarray
    flow_value: np.ndarray
    flow_off: np.ndarray
    flow_times: np.ndarray
    flow_vals: np.ndarray
    other_idx: np.ndarray
    other_type: np.ndarray
    other_value: np.ndarray
    other_off: np.ndarray
    other_times: np.ndarray
    other_vals: np.ndarray
    rain_times: np.ndarray
    rain_rates: np.ndarray

    @property
    def n_flow(self) -> int:
        return int(self.flow_idx.size)

    @property
    def n_other(self) -> int:
        return int(self.other_idx.size)

    @property
    def n_rain(self) -> int:
        return int(self.rain_times.size)


def _csr(points: List[sc.PointBC]):
    off = np.zeros(len(points) + 1, dtype=np.int32)
    times, vals = [], []
    for k, p in enumerate(points):
        n = 0
        if p.kind in (sc.QVAR, sc.HVAR) and p.times is not None:
            times.append(np.asarray(p.times, dtype=np.float64))
            vals.append(np.asarray(p.values, dtype=np.float64))
            n = len(p.times)
        off[k + 1] = off[k] + n
    t = np.concatenate(times) if times else np.zeros(0)
    v = np.concatenate(vals) if vals else np.zeros(0)
    return off, t, v


_OTHER_DEVICE_TYPE = {sc.FREE: 1, sc.HFIX: 2, sc.HVAR: 3}


def pack(case: sc.Case) -> Forcing:
    flow = case.flow_points()
    other = case.other_points()
    fo, ft, fv = _csr(flow)
    oo, ot, ov = _csr(other)
    nx = case.nx
    if case.rain_times is not None and len(case.rain_times):
        rt = np.asarray(case.rain_times, dtype=np.float64)
        rr = np.asarray(case.rain_rates, dtype=np.float64)
    else:
        rt = np.zeros(0)
        rr = np.zeros(0)
    return Forcing(
        flow_idx=np.array([p.i + p.j * nx for p in flow], dtype=np.int32),
        flow_type=np.array([p.kind for p in flow], dtype=np.int32),
        flow_value=np.array([p.value if p.kind == sc.QFIX else 0.0 for p in flow],
                            dtype=np.float64),
        flow_off=fo, flow_times=ft, flow_vals=fv,
        other_idx=np.array([p.i + p.j * nx for p in other], dtype=np.int32),
        other_type=np.array([_OTHER_DEVICE_TYPE[p.kind] for p in other], dtype=np.int32),
        other_value=np.array([p.value if p.kind == sc.HFIX else 0.0 for p in other],
                             dtype=np.float64),
        other_off=oo, other_times=ot, other_vals=ov,
        rain_times=rt, rain_rates=rr,
    )
