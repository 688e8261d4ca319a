"""The run with the reference's file outputs (af_sim_run_output) against the
reference's own CLI (its src/main.cpp, compiled against the Kokkos-API shim)
on the same case: the same files, identical headers, values within the last
printed digit (FP64 depths agree to 1e-9 m; a value within 1e-9 of a rounding
boundary of "%.4f" may print one unit apart), the same stage.csv."""
import os
import subprocess

import numpy as np
import pytest

from adaptflood_b200 import scenarios as sc
from adaptflood_b200.sim import Simulation
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _case():
    c = sc.small_case(70, 50, seed=51, rain=True, n_hvar=1, n_free_pts=1, sim_time=300.0)
    c.save_int, c.mass_int = 60.0, 60.0
    c.xll, c.yll = 1000.0, 2000.5
    return c


STAGES = [("gauge_a", 10, 12), ("gauge_b", 35, 25), ("outside", 5, 80)]


def _run_reference(case, tmp, voutput, async_out):
    d = os.path.join(tmp, "ref_in")
    out = os.path.join(tmp, "ref_out")
    par = case.write(d, out_dir=out)
    stage_path = os.path.join(d, "stages.txt")
    with open(stage_path, "w") as f:
        for name, i, j in STAGES:
            x = case.xll + (i + 0.5) * case.dx
            y = case.yll + case.ny * case.dx - (j + 0.5) * case.dx
            f.write(f"{x!r} {y!r} {name}\n")
    with open(par, "a") as f:
        f.write(f"stagefile {stage_path}\nstageint 30\n")
        f.write(f"async_output {int(async_out)}\n")
        if voutput:
            f.write("voutput 1\n")
    # The reference opens stage.csv before it creates dirroot (src/main.cpp:100
    # versus :130), so it only writes stage output into an existing directory.
    os.makedirs(out, exist_ok=True)
    subprocess.run([orc.REF_CLI, par], cwd=tmp, check=True, capture_output=True, timeout=300)
    return out


def _read_asc(path):
    lines = open(path).read().splitlines()
    return lines[:6], [row.split() for row in lines[6:]]


@pytest.mark.parametrize("voutput,async_out", [(True, True), (False, False), (True, False)])
def test_outputs_match_reference_cli(cuda, tmp_path, voutput, async_out):
    if not os.path.exists(orc.REF_CLI):
        pytest.skip("reference CLI not built")
    case = _case()
    ref_dir = _run_reference(case, str(tmp_path), voutput, async_out)
    ours = str(tmp_path / "ours")
    with Simulation(case, "f64") as s:
        s.run_output(ours, voutput=voutput, async_style=async_out, stages=STAGES, stage_int=30.0)
    _compare_with_reference(case, ref_dir, ours)


def test_par_file_run_matches_reference_cli(cuda, tmp_path):
    """The same .par file run by run_par (inputs, outputs and stage points all
    read by this library, af_scenario_output) and by the reference's CLI
    gives the same files."""
    if not os.path.exists(orc.REF_CLI):
        pytest.skip("reference CLI not built")
    from adaptflood_b200.sim import run_par
    case = _case()
    ref_dir = _run_reference(case, str(tmp_path), True, True)
    par = os.path.join(str(tmp_path), "ref_in", "case.par")
    ours = str(tmp_path / "ours")
    mine = os.path.join(str(tmp_path), "mine.par")
    with open(par) as f, open(mine, "w") as g:
        for line in f:
            g.write(f"dirroot {ours}\n" if line.startswith("dirroot") else line)
    os.makedirs(ours, exist_ok=True)
    run_par(mine, "f64")
    _compare_with_reference(case, ref_dir, ours)


def _compare_with_reference(case, ref_dir, ours):
    ref_files = sorted(f for f in os.listdir(ref_dir) if f.endswith((".asc", ".csv")))
    our_files = sorted(os.listdir(ours))
    assert our_files == ref_files
    assert "H_final.asc" in our_files and "H_0005.asc" in our_files
    for name in ref_files:
        if name == "stage.csv":
            continue
        hr, vr = _read_asc(os.path.join(ref_dir, name))
        ho, vo = _read_asc(os.path.join(ours, name))
        assert ho == hr, name
        a = np.array(vr, dtype=np.float64)
        b = np.array(vo, dtype=np.float64)
        assert a.shape == b.shape == (case.ny, case.nx)
        assert np.max(np.abs(a - b)) <= 1.01e-4, name
        same = np.mean(np.array(vr) == np.array(vo))
        assert same >= 0.995, (name, same)
    sr = open(os.path.join(ref_dir, "stage.csv")).read().splitlines()
    so = open(os.path.join(ours, "stage.csv")).read().splitlines()
    assert so[0] == sr[0] and len(so) == len(sr) > 5
    for lr, lo in zip(sr[1:], so[1:]):
        fr, fo = lr.split(","), lo.split(",")
        assert fo[0] == fr[0] and fo[-1] == fr[-1] == "NaN"
        assert np.allclose([float(x) for x in fo[1:-1]], [float(x) for x in fr[1:-1]],
                           atol=1.01e-4, rtol=0)


def test_fp32_output_run_matches_fp64_within_tolerance(cuda, tmp_path):
    case = _case()
    for prec in ("f64", "f32"):
        with Simulation(case, prec) as s:
            s.run_output(str(tmp_path / prec), voutput=True)
    _, a = _read_asc(str(tmp_path / "f64" / "H_final.asc"))
    _, b = _read_asc(str(tmp_path / "f32" / "H_final.asc"))
    assert np.max(np.abs(np.array(a, float) - np.array(b, float))) <= 1e-3 + 1e-4


@pytest.mark.parametrize("fmt", [1, 2])
def test_netcdf_output(cuda, tmp_path, fmt):
    """With the async writer and output_format 1 (NetCDF) or 2 (both), every
    save is a record of output.nc with the reference's schema
    (src/async_output.cpp:20-51: dimensions time/x/y, time in seconds, H, Vx,
    Vy as float with their attributes, the georeference as global
    attributes); the records hold the saved fields rounded to float, the last
    one the final state.  Format 1 writes no periodic ASC grids, only the
    final ones."""
    from scipy.io import netcdf_file
    case = _case()  # 300 s, saves every 60 s: the start and five more
    out = str(tmp_path / "nc")
    with Simulation(case, "f64") as s:
        s.run_output(out, voutput=True, async_style=True, output_format=fmt)
        t_end = s.status()[0]
        H = s.depth()
        Vx, Vy = s.velocity()
    files = sorted(os.listdir(out))
    assert "output.nc" in files and "H_final.asc" in files and "Vx_final.asc" in files
    assert ("H_0003.asc" in files) == (fmt == 2)
    with netcdf_file(os.path.join(out, "output.nc"), "r", mmap=False) as f:
        assert f.version_byte == 2
        assert f.dimensions["time"] is None
        assert f.dimensions["x"] == case.nx and f.dimensions["y"] == case.ny
        assert (f.xllcorner, f.yllcorner, f.cellsize) == (case.xll, case.yll, case.dx)
        tv, hv, vx, vy = (f.variables[k] for k in ("time", "H", "Vx", "Vy"))
        assert tv.units == b"seconds"
        assert hv.units == b"m" and hv.long_name == b"water_depth"
        assert hv._FillValue == np.float32(case.nodata)
        assert vx.units == vy.units == b"m/s"
        assert vx.long_name == b"x_direction_velo" and vy.long_name == b"y_direction_velo"
        assert hv.dimensions == vx.dimensions == ("time", "y", "x")
        times = tv[:].copy()
        assert len(times) == 6 and times[0] == 0.0 and times[-1] == t_end
        assert np.all(np.diff(times) > 0) and np.all(times[1:] >= 60.0 * np.arange(1, 6))
        assert hv.shape == (6, case.ny, case.nx)
        np.testing.assert_array_equal(hv[0], np.zeros((case.ny, case.nx), np.float32))
        np.testing.assert_array_equal(hv[5], H.astype(np.float32))
        np.testing.assert_array_equal(vx[5], Vx.astype(np.float32))
        np.testing.assert_array_equal(vy[5], Vy.astype(np.float32))
        if fmt == 2:
            _, a = _read_asc(os.path.join(out, "H_0003.asc"))
            assert np.max(np.abs(np.array(a, float) - hv[3].astype(float))) <= 5.01e-5 + 1e-6
