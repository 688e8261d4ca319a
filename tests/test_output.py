"""The reference's file outputs: ESRI ASCII grids with printf("%.4f ")
values in the headers of its two writers, and its NetCDF file (host code, no
device)."""
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


def _nc_create(path, nx, ny, voutput, xll=1000.0, yll=2000.5, cs=2.0, nd=-9999.0):
    h = C.c_void_p()
    rc = _lib.lib().af_netcdf_create(str(path).encode(), nx, ny, int(voutput), xll, yll, cs, nd,
                                     C.byref(h))
    assert rc == _lib.AF_OK
    return h


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def test_netcdf_writer_schema_and_records(tmp_path):
    """The reference's NetCDF schema (src/async_output.cpp:20-51) read back by
    SciPy's independent NetCDF reader; records of more than one write chunk
    (1.1 M cells); values rounded to float; the record count is in the file
    after every record."""
    from scipy.io import netcdf_file
    lib = _lib.lib()
    nx, ny = 1100, 1000
    rng = np.random.default_rng(9)
    path = tmp_path / "output.nc"
    h = _nc_create(path, nx, ny, True)
    recs = []
    try:
        for k, t in enumerate((0.0, 600.25, 1200.5)):
            H, Vx, Vy = (rng.normal(0, 2, (ny, nx)) for _ in range(3))
            assert lib.af_netcdf_append(h, t, _p(H), _p(Vx), _p(Vy)) == _lib.AF_OK
            recs.append((t, H, Vx, Vy))
            with netcdf_file(str(path), "r", mmap=False) as f:
                assert f.variables["time"].shape == (k + 1,)
    finally:
        assert lib.af_netcdf_close(h) == _lib.AF_OK
    with netcdf_file(str(path), "r", mmap=False) as f:
        assert f.version_byte == 2
        assert f.dimensions["time"] is None
        assert (f.dimensions["x"], f.dimensions["y"]) == (nx, ny)
        assert (f.xllcorner, f.yllcorner, f.cellsize) == (1000.0, 2000.5, 2.0)
        assert list(f.variables) == ["time", "H", "Vx", "Vy"]
        assert f.variables["H"].dimensions == ("time", "y", "x")
        assert f.variables["H"].long_name == b"water_depth"
        assert f.variables["H"]._FillValue == np.float32(-9999.0)
        assert f.variables["Vy"].long_name == b"y_direction_velo"
        assert f.variables["H"].data.dtype.kind == "f" and f.variables["H"].data.itemsize == 4
        np.testing.assert_array_equal(f.variables["time"][:], [r[0] for r in recs])
        for k, (t, H, Vx, Vy) in enumerate(recs):
            np.testing.assert_array_equal(f.variables["H"][k], H.astype(np.float32))
            np.testing.assert_array_equal(f.variables["Vx"][k], Vx.astype(np.float32))
            np.testing.assert_array_equal(f.variables["Vy"][k], Vy.astype(np.float32))


def test_netcdf_writer_depth_only_and_errors(tmp_path):
    from scipy.io import netcdf_file
    lib = _lib.lib()
    path = tmp_path / "d.nc"
    h = _nc_create(path, 7, 5, False)
    H = np.arange(35, dtype=np.float64).reshape(5, 7) / 3.0
    assert lib.af_netcdf_append(h, 60.0, _p(H), None, None) == _lib.AF_OK
    assert lib.af_netcdf_close(h) == _lib.AF_OK
    with netcdf_file(str(path), "r", mmap=False) as f:
        assert list(f.variables) == ["time", "H"]
        np.testing.assert_array_equal(f.variables["H"][0], H.astype(np.float32))
    out = C.c_void_p()
    assert lib.af_netcdf_create(None, 7, 5, 0, 0.0, 0.0, 1.0, -9999.0, C.byref(out)) == _lib.AF_EINVAL
    assert lib.af_netcdf_create(b"x.nc", 0, 5, 0, 0.0, 0.0, 1.0, -9999.0, C.byref(out)) == _lib.AF_EINVAL
    assert lib.af_netcdf_create(b"x.nc", 40000, 40000, 0, 0.0, 0.0, 1.0, -9999.0,
                                C.byref(out)) == _lib.AF_ERANGE
    h = _nc_create(tmp_path / "v.nc", 7, 5, True)
    assert lib.af_netcdf_append(h, 0.0, _p(H), None, None) == _lib.AF_EINVAL
    assert lib.af_netcdf_close(h) == _lib.AF_OK
