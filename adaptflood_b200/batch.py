"""Python host API over the batch layer (af_batch_* in include/adaptflood.h).

A :class:`Batch` holds many independent flood scenarios (grids of uneven
sizes, each with its own parameters, forcing, adaptive dt and stop time) in
one device arena and steps them together: one persistent kernel per batch
step inside one CUDA graph.  Each scenario evolves exactly as a
:class:`adaptflood_b200.sim.Simulation` of the same case and precision would
alone; its stop time plays the role of the reference's ``sim_time``
(src/main.cpp:227).

Admission is by device-memory footprint: :meth:`Batch.try_add` returns
``None`` when the scenario does not fit in the free arena space (nothing
changes), so a caller can queue it and retry after :meth:`Batch.remove`.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Tuple

import numpy as np

from . import _lib
from . import forcing as fc
from . import scenarios as sc
from .sim import _ForcingArrays, _p, case_desc

PRECISIONS = {"f64": _lib.AF_PREC_F64, "f32": _lib.AF_PREC_F32}
RUNNING, FINISHED, FAILED = 0, 1, -1


def size_class(nx: int, ny: int) -> int:
    """floor(log2(nx*ny)): the key of the strip-height table."""
    return _lib.lib().af_batch_size_class(int(nx), int(ny))


class Batch:
    def __init__(self, precision: str = "f32", device: int = 0,
                 arena_bytes: Optional[int] = None, variant: int = -1,
                 rows: Optional[Dict[int, int]] = None):
        self.lib = _lib.lib()
        self.precision = precision
        if arena_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            arena_bytes = int(free * 0.8)
        self.arena_bytes = int(arena_bytes)
        h = C.c_void_p()
        _lib.check(self.lib.af_batch_create(PRECISIONS[precision], device, self.arena_bytes,
                                            variant, C.byref(h)), "af_batch_create")
        self.h = h
        self.cases: Dict[int, sc.Case] = {}
        for cls, r in (rows or {}).items():
            self.set_rows(cls, r)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.af_batch_destroy(self.h)
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

    # ------------------------------------------------------------ shapes
    def set_rows(self, cls: int, rows: int) -> None:
        _lib.check(self.lib.af_batch_set_rows(self.h, int(cls), int(rows)), "af_batch_set_rows")

    def set_balance(self, strips_per_warp: int) -> None:
        """Load-adaptive strip height target (0 = off); see af_batch_set_balance."""
        _lib.check(self.lib.af_batch_set_balance(self.h, int(strips_per_warp)),
                   "af_batch_set_balance")

    def rows(self, cls: int) -> int:
        return self.lib.af_batch_get_rows(self.h, int(cls))

    # --------------------------------------------------------- admission
    def footprint(self, case: sc.Case, forcing: Optional[fc.Forcing] = None,
                  t_stop: Optional[float] = None) -> int:
        f = _ForcingArrays(forcing if forcing is not None else fc.pack(case))
        d = case_desc(case)
        n = C.c_uint64()
        t = case.sim_time if t_stop is None else t_stop
        _lib.check(self.lib.af_batch_footprint(self.h, C.byref(d), C.byref(f.desc), float(t),
                                               C.byref(n)), "af_batch_footprint")
        return n.value

    def try_add(self, case: sc.Case, forcing: Optional[fc.Forcing] = None,
                t_stop: Optional[float] = None) -> Optional[int]:
        """Admits a scenario; returns its slot, or None when the arena (or the
        slot table) has no room for it."""
        f = _ForcingArrays(forcing if forcing is not None else fc.pack(case))
        d = case_desc(case)
        dem = np.ascontiguousarray(case.dem, dtype=np.float64)
        h0 = None if case.h0 is None else np.ascontiguousarray(case.h0, dtype=np.float64)
        t = case.sim_time if t_stop is None else t_stop
        slot = C.c_int(-1)
        rc = self.lib.af_batch_add(self.h, C.byref(d), C.byref(f.desc), _p(dem), _p(h0), float(t),
                                   C.byref(slot))
        if rc == _lib.AF_ENOMEM:
            return None
        _lib.check(rc, "af_batch_add")
        self.cases[slot.value] = case
        return slot.value

    def add(self, case: sc.Case, forcing: Optional[fc.Forcing] = None,
            t_stop: Optional[float] = None) -> int:
        s = self.try_add(case, forcing, t_stop)
        if s is None:
            raise _lib.AFError(_lib.AF_ENOMEM, "af_batch_add")
        return s

    def remove(self, slot: int) -> None:
        _lib.check(self.lib.af_batch_remove(self.h, int(slot)), "af_batch_remove")
        self.cases.pop(slot, None)

    # ---------------------------------------------------------- stepping
    def launch(self, max_steps: int = 1 << 40, stop_on_done: bool = False) -> None:
        _lib.check(self.lib.af_batch_launch(self.h, int(max_steps), int(stop_on_done)),
                   "af_batch_launch")

    def attention(self) -> None:
        _lib.check(self.lib.af_batch_attention(self.h), "af_batch_attention")

    def done(self) -> bool:
        """True when no launch is in flight or it has finished (never waits)."""
        rc = self.lib.af_batch_query(self.h)
        if rc < 0:
            _lib.check(rc, "af_batch_query")
        return rc == 1

    def sync(self) -> None:
        _lib.check(self.lib.af_batch_sync(self.h), "af_batch_sync")

    def run(self, max_steps: int = 1 << 40) -> int:
        """Steps until every member has finished (or max_steps batch steps)."""
        n = C.c_int64()
        _lib.check(self.lib.af_batch_run(self.h, int(max_steps), C.byref(n)), "af_batch_run")
        return n.value

    @property
    def stream(self) -> int:
        return self.lib.af_batch_stream(self.h) or 0

    # ------------------------------------------------------------ results
    def status(self, slot: int) -> Tuple[float, float, float, int, int]:
        """(t, dt_last, hmax, steps, state) as of the last sync."""
        t, dt, hm = C.c_double(), C.c_double(), C.c_double()
        n, st = C.c_int64(), C.c_int()
        _lib.check(self.lib.af_batch_slot_status(self.h, int(slot), C.byref(t), C.byref(dt),
                                                 C.byref(hm), C.byref(n), C.byref(st)),
                   "af_batch_slot_status")
        return t.value, dt.value, hm.value, n.value, st.value

    def state(self, slot: int) -> dict:
        case = self.cases[slot]
        nx, ny = case.nx, case.ny
        H = np.zeros(nx * ny)
        Qx = np.zeros((nx + 1) * (ny + 1))
        Qy = np.zeros((nx + 1) * (ny + 1))
        _lib.check(self.lib.af_batch_get_state(self.h, int(slot), _p(H), _p(Qx), _p(Qy)),
                   "af_batch_get_state")
        return {"H": H.reshape(ny, nx), "Qx": Qx.reshape(ny + 1, nx + 1),
                "Qy": Qy.reshape(ny + 1, nx + 1)}

    def depth(self, slot: int) -> np.ndarray:
        case = self.cases[slot]
        H = np.zeros(case.nx * case.ny)
        _lib.check(self.lib.af_batch_get_state(self.h, int(slot), _p(H), None, None),
                   "af_batch_get_state")
        return H.reshape(case.ny, case.nx)

    def mass_series(self, slot: int):
        n = C.c_int()
        _lib.check(self.lib.af_batch_mass_series(self.h, int(slot), None, None, None, 0,
                                                 C.byref(n)), "af_batch_mass_series")
        k = n.value
        t, v, a = np.zeros(max(k, 1)), np.zeros(max(k, 1)), np.zeros(max(k, 1))
        _lib.check(self.lib.af_batch_mass_series(self.h, int(slot), _p(t), _p(v), _p(a), k,
                                                 C.byref(n)), "af_batch_mass_series")
        return t[:k], v[:k], a[:k]

    def set_trace(self, cap: int) -> None:
        """Records up to `cap` batch steps from now (0: off); see trace()."""
        _lib.check(self.lib.af_batch_set_trace(self.h, int(cap)), "af_batch_set_trace")

    def trace(self) -> np.ndarray:
        """The recorded steps since set_trace, one row each: start and end on
        the device clock (ns), cells and strips stepped."""
        n = C.c_int64()
        _lib.check(self.lib.af_batch_get_trace(self.h, None, 0, C.byref(n)), "af_batch_get_trace")
        out = np.zeros((max(n.value, 1), 4), dtype=np.int64)
        _lib.check(self.lib.af_batch_get_trace(self.h, _p(out), n.value, C.byref(n)),
                   "af_batch_get_trace")
        return out[:n.value]

    def info(self) -> dict:
        m = C.c_int()
        st = C.c_int64()
        ab, au, al = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _lib.check(self.lib.af_batch_info(self.h, C.byref(m), C.byref(st), C.byref(ab),
                                          C.byref(au), C.byref(al)), "af_batch_info")
        return {"members": m.value, "batch_steps": st.value, "arena_bytes": ab.value,
                "arena_used": au.value, "arena_largest_free": al.value}


class Arena:
    """The batch's arena planner on the host (no device memory)."""

    def __init__(self, nbytes: int):
        self.lib = _lib.lib()
        h = C.c_void_p()
        _lib.check(self.lib.af_arena_create(int(nbytes), C.byref(h)), "af_arena_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.af_arena_destroy(self.h)
            self.h = None

    def alloc(self, nbytes: int) -> Optional[int]:
        off = C.c_uint64()
        rc = self.lib.af_arena_alloc(self.h, int(nbytes), C.byref(off))
        if rc == _lib.AF_ENOMEM:
            return None
        _lib.check(rc, "af_arena_alloc")
        return off.value

    def free(self, off: int) -> None:
        _lib.check(self.lib.af_arena_free(self.h, int(off)), "af_arena_free")

    def stats(self) -> Tuple[int, int, int]:
        u, lf, b = C.c_uint64(), C.c_uint64(), C.c_int()
        _lib.check(self.lib.af_arena_stats(self.h, C.byref(u), C.byref(lf), C.byref(b)),
                   "af_arena_stats")
        return u.value, lf.value, b.value


def trace_summary(rec: np.ndarray, bytes_per_cell: float, peak_gbs: float) -> dict:
    """Where a traced batch run spent its time: steps grouped by the cells
    they stepped (powers of four), each group's share of the time and of the
    cell-updates, and its HBM rate (algorithmic bytes / device time)."""
    if rec.size == 0:
        return {}
    start, end, cells, _units = (rec[:, k].astype(np.float64) for k in range(4))
    dt = (end - start) * 1e-9
    total = float(dt.sum())
    cu = float(cells.sum())
    edges = [0.0] + [float(4 ** k) for k in range(8, 15)] + [np.inf]
    groups = []
    for lo, hi in zip(edges[:-1], edges[1:]):
        m = (cells >= lo) & (cells < hi)
        if not m.any():
            continue
        t = float(dt[m].sum())
        c = float(cells[m].sum())
        groups.append({"cells": [lo, hi if np.isfinite(hi) else None], "steps": int(m.sum()),
                       "time_share": t / total, "cell_update_share": c / cu,
                       "hbm_frac": (c * bytes_per_cell / t / 1e9) / peak_gbs if t > 0 else None,
                       "us_per_step": t / int(m.sum()) * 1e6})
    return {"steps": int(rec.shape[0]), "seconds": total,
            "min_step_us": float(dt.min() * 1e6), "groups": groups}

