"""Pins the CPU oracle (oracle/af_oracle.c) to the reference.

* against the committed golden fixtures, which the reference's own
  src/kernels.cpp + src/main.cpp loop produced (tests/golden/make_golden.py);
* against the reference library itself on freshly generated cases, where
  oracle/_ref is present.
The bar is bit-exactness: same dt series, same fields, to the last bit.
"""
import math

import numpy as np
import pytest

from _util import golden_names, load_golden
from adaptflood_b200 import forcing as fc
from adaptflood_b200 import scenarios as sc
from oracle import oracle as orc


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_golden(name):
    case, f, exp = load_golden(name)
    o = orc.OracleSim(case, f)
    dts = o.run(case.sim_time, record_dt=True)
    np.testing.assert_array_equal(dts, exp["dt"])
    assert o.t == float(exp["t_end"])
    st = o.state(velocity=True)
    for k in ("H", "Qx", "Qy", "Vx", "Vy"):
        np.testing.assert_array_equal(st[k], exp[k], err_msg=k)


@pytest.mark.parametrize("name", golden_names())
def test_golden_inputs_parse_as_generated(name):
    """The reference parsed the generated files into exactly the tables the
    generator packed (so the oracle/GPU inputs are the reference's inputs)."""
    case, f, exp = load_golden(name)
    assert tuple(bool(x) for x in exp["ref_free"]) == (case.west_free, case.east_free,
                                                       case.north_free, case.south_free)
    idx = np.concatenate([f.flow_idx, f.other_idx])
    np.testing.assert_array_equal(exp["ref_pt_idx"], idx)
    # reference BoundaryType: QFIX 4, QVAR 5, FREE 1, HFIX 2, HVAR 3
    other_bt = np.array([{1: 1, 2: 2, 3: 3}[t] for t in f.other_type], dtype=np.int32)
    np.testing.assert_array_equal(exp["ref_pt_type"], np.concatenate([f.flow_type, other_bt]))
    np.testing.assert_array_equal(exp["ref_pt_value"], np.concatenate([f.flow_value, f.other_value]))
    nser = np.concatenate([np.diff(f.flow_off), np.diff(f.other_off)])
    np.testing.assert_array_equal(exp["ref_pt_nser"], nser)


def test_golden_cover_the_features():
    names = golden_names()
    assert len(names) >= 6
    feats = set()
    for n in names:
        case, f, _ = load_golden(n)
        feats |= {"rain"} if f.n_rain else set()
        feats |= {"nodata"} if np.any(case.dem == case.nodata) else set()
        feats |= {"h0"} if case.h0 is not None else set()
        feats |= {"closed"} if not case.west_free else {"west_free"}
        feats |= {"qfix"} if np.any(f.flow_type == sc.QFIX) else set()
        feats |= {"qvar"} if np.any(f.flow_type == sc.QVAR) else set()
        feats |= {"hfix"} if np.any(f.other_type == 2) else set()
        feats |= {"hvar"} if np.any(f.other_type == 3) else set()
        feats |= {"free_pt"} if np.any(f.other_type == 1) else set()
        feats |= {"dup"} if len(set(f.flow_idx.tolist())) < f.n_flow else set()
        feats |= {"nx2"} if case.nx == 2 else set()
    assert feats >= {"rain", "nodata", "h0", "closed", "west_free", "qfix", "qvar", "hfix",
                     "hvar", "free_pt", "dup", "nx2"}


LIVE = [
    dict(nx=29, ny=23, seed=101, kw=dict(rain=True, n_hvar=2, dup_sources=True)),
    dict(nx=17, ny=41, seed=102, kw=dict(free=(0, 1, 1, 0), nodata_block=True, n_free_pts=2)),
    dict(nx=45, ny=12, seed=103, kw=dict(free=(1, 1, 0, 0), h0=True, n_hfix=2)),
]


@pytest.mark.parametrize("spec", LIVE, ids=lambda s: f"{s['nx']}x{s['ny']}")
def test_oracle_matches_reference_live(spec, tmp_path):
    if not orc.ref_available():
        pytest.skip("reference library not built here")
    case = sc.small_case(spec["nx"], spec["ny"], seed=spec["seed"], sim_time=200.0, **spec["kw"])
    r = orc.RefSim(case.write(str(tmp_path)))
    if case.h0 is not None:
        r.set_h(case.h0.ravel())
    o = orc.OracleSim(case, fc.pack(case))
    np.testing.assert_array_equal(r.run(case.sim_time, record_dt=True),
                                  o.run(case.sim_time, record_dt=True))
    a, b = r.state(), o.state()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def _interp_py(times, vals, fixed, t):
    """src/io.cpp:299-311 written out in Python."""
    n = len(times)
    if n == 0:
        return fixed
    if t <= times[0]:
        return vals[0]
    if t >= times[-1]:
        return vals[-1]
    for i in range(n - 1):
        if times[i] <= t < times[i + 1]:
            ratio = (t - times[i]) / (times[i + 1] - times[i])
            return vals[i] + ratio * (vals[i + 1] - vals[i])
    return vals[-1]


def test_interp_semantics():
    import ctypes as C
    lib = orc._oracle_lib()
    lib.afo_interp.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double]
    cases = [
        ([], [], 0.7, 5.0),
        ([0.0, 60.0, 60.0, 120.0], [1.0, 1.0, 3.0, 3.0], 0, 60.0),  # repeated time: step
        ([0.0, 60.0, 60.0, 120.0], [1.0, 1.0, 3.0, 3.0], 0, 59.999),
        ([10.0, 20.0], [2.0, 4.0], 0, 5.0),
        ([10.0, 20.0], [2.0, 4.0], 0, 25.0),
        ([10.0, 20.0], [2.0, 4.0], 0, 12.5),
        ([0.0, 30.0, 10.0], [0.0, 3.0, 1.0], 0, 20.0),  # unsorted: falls through
        ([0.0, 10.0], [0.0, 1.0], 0, float("nan")),
    ]
    for times, vals, fixed, t in cases:
        tt = np.array(times, dtype=np.float64)
        vv = np.array(vals, dtype=np.float64)
        got = lib.afo_interp(tt.ctypes.data, vv.ctypes.data, len(times), float(fixed), t)
        want = _interp_py(times, vals, fixed, t)
        assert (got == want) or (math.isnan(got) and math.isnan(want)), (times, t, got, want)
