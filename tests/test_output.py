"""The reference's file outputs: ESRI ASCII grids with printf("%.4f ")
values in the headers of its two writers (host code, no device)."""
import ctypes as C

import numpy as np
import pytest

from adaptflood_b200 import _lib

HEAD = {
    0: "ncols         {nx}\nnrows         {ny}\nxllcorner     {xll:.1f}\nyllcorner     {yll:.1f}\n"
       "cellsize      {cs:.1f}\nNODATA_value  -9999\n",
    1: "ncols         {nx}\nnrows         {ny}\nxllcorner     {xll:.6f}\nyllcorner     {yll:.6f}\n"
       "cellsize      {cs:.1f}\nNODATA_value  {nd:.0f}\n",
}


def _expected(v, style, xll, yll, cs, nd):
    ny, nx = v.shape
    out = HEAD[style].format(nx=nx, ny=ny, xll=xll, yll=yll, cs=cs, nd=nd)
    for row in v:
        out += "".join("%.4f " % x for x in row) + "\n"
    return out


def _write(tmp_path, v, style, xll=12.5, yll=-3.25, cs=5.0, nd=-9999.0):
    path = str(tmp_path / f"g{style}.asc")
    a = np.ascontiguousarray(v, dtype=np.float64)
    rc = _lib.lib().af_write_asc(path.encode(), a.ctypes.data_as(C.c_void_p), a.shape[1],
                                 a.shape[0], xll, yll, cs, nd, style)
    assert rc == _lib.AF_OK
    return open(path).read(), _expected(v, style, xll, yll, cs, nd)


# printf rounds the exact binary value: ties (k + 1/2) * 1e-4 that doubles hold
# exactly go to even, and values that round to zero keep their sign.
EDGE = [0.0, -0.0, 0.03125, 0.09375, 0.15625, 1.03125, 2.5e-5, -2.5e-5, 5e-5, 1.5e-4, 0.00005,
        -0.00001, -0.00004999, 0.99995, 0.999949999, 9.99995, 1234.56785, -7.00005, 1e10,
        123456789.01235, 0.1, 0.2, 0.3, 1e-300, 3.0000499999999997, 2.00015, 62.5 / 1e4]


@pytest.mark.parametrize("style", [0, 1])
def test_edge_values_match_printf(tmp_path, style):
    v = np.array(EDGE + [0.0] * (-len(EDGE) % 9), dtype=np.float64).reshape(-1, 9)
    got, want = _write(tmp_path, v, style)
    assert got == want


def test_random_values_match_printf(tmp_path):
    rng = np.random.default_rng(3)
    v = np.concatenate([rng.uniform(-5, 5, 20000), rng.exponential(0.01, 20000),
                        np.round(rng.uniform(0, 100, 20000), 5),
                        rng.integers(0, 2000000, 20000) / 20000.0,  # many exact halves of 1e-4
                        -rng.exponential(1e-5, 20000)]).reshape(500, 200)
    got, want = _write(tmp_path, v, 1, xll=0.0, yll=0.0, cs=10.0)
    assert got == want


def test_large_grid_written_in_parallel_blocks(tmp_path):
    rng = np.random.default_rng(4)
    v = rng.uniform(0, 3, size=(700, 640))  # above the parallel-formatting threshold
    got, want = _write(tmp_path, v, 0)
    assert got == want


def test_invalid_arguments(tmp_path):
    lib = _lib.lib()
    assert lib.af_write_asc(None, None, 1, 1, 0.0, 0.0, 1.0, -9999.0, 0) == _lib.AF_EINVAL
    assert lib.af_write_asc(b"x", None, 2, 2, 0.0, 0.0, 1.0, -9999.0, 0) == _lib.AF_EINVAL
    a = np.zeros(4)
    assert lib.af_write_asc(str(tmp_path / "a.asc").encode(), a.ctypes.data_as(C.c_void_p),
                            2, 2, 0.0, 0.0, 1.0, -9999.0, 7) == _lib.AF_EINVAL
    assert lib.af_write_asc(b"/nonexistent-dir/a.asc", a.ctypes.data_as(C.c_void_p), 2, 2,
                            0.0, 0.0, 1.0, -9999.0, 0) == _lib.AF_EIO
