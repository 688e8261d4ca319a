"""The library's input readers (af_scenario_load) against the generator and
against the reference's own parsers, including the reference's quirks."""
import os

import numpy as np
import pytest

from adaptflood_b200 import _lib
from adaptflood_b200 import forcing as fc
from adaptflood_b200 import scenarios as sc
from adaptflood_b200.sim import load_par
from oracle import oracle as orc


def _assert_forcing_equal(a: fc.Forcing, b: fc.Forcing):
    for k in a.__dataclass_fields__:
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)


@pytest.mark.parametrize("seed,kw", [
    (1, dict()),
    (2, dict(rain=True, n_hfix=2, n_hvar=1, n_free_pts=2, dup_sources=True, nodata_block=True)),
    (3, dict(free=(0, 1, 0, 1), n_qvar=4)),
])
def test_reader_matches_generator(tmp_path, seed, kw):
    case = sc.small_case(23, 19, seed=seed, sim_time=321.5, **kw)
    par = case.write(str(tmp_path))
    got, f = load_par(par)
    assert (got.nx, got.ny, got.dx, got.nodata) == (case.nx, case.ny, case.dx, case.nodata)
    np.testing.assert_array_equal(got.dem, case.dem)
    assert (got.west_free, got.east_free, got.north_free, got.south_free) == (
        case.west_free, case.east_free, case.north_free, case.south_free)
    assert (got.sim_time, got.save_int, got.mass_int, got.cfl, got.fpn, got.depth_thresh,
            got.init_tstep) == (case.sim_time, case.save_int, case.mass_int, case.cfl, case.fpn,
                                case.depth_thresh, case.init_tstep)
    _assert_forcing_equal(f, fc.pack(case))


def test_reader_matches_reference_parse(tmp_path):
    if not orc.ref_available():
        pytest.skip("reference library not built here")
    case = sc.small_case(31, 27, seed=9, rain=True, n_hfix=1, n_hvar=2, n_free_pts=1,
                         dup_sources=True, free=(1, 0, 0, 1))
    par = case.write(str(tmp_path))
    _, f = load_par(par)
    r = orc.RefSim(par)
    idx, typ, val, nser = r.points()
    np.testing.assert_array_equal(idx, np.concatenate([f.flow_idx, f.other_idx]))
    np.testing.assert_array_equal(val, np.concatenate([f.flow_value, f.other_value]))
    np.testing.assert_array_equal(nser, np.concatenate([np.diff(f.flow_off), np.diff(f.other_off)]))
    assert r.free == (case.west_free, case.east_free, case.north_free, case.south_free)
    assert r.rain_enabled == (f.n_rain > 0)


def _minimal(tmp_path, bci: str, bdy: str = "title\n", rain: str = None, dem_rows=None):
    d = str(tmp_path)
    dem_rows = dem_rows or ["1 2 3", "4 5 6"]
    with open(os.path.join(d, "dem.asc"), "w") as fh:
        fh.write("ncols 3\nnrows 2\nxllcorner 0\nyllcorner 0\ncellsize 10\nNODATA_value -9999\n")
        fh.write("\n".join(dem_rows) + "\n")
    with open(os.path.join(d, "c.bci"), "w") as fh:
        fh.write(bci)
    with open(os.path.join(d, "c.bdy"), "w") as fh:
        fh.write(bdy)
    lines = [f"DEMfile {d}/dem.asc", f"bcifile {d}/c.bci", f"bdyfile {d}/c.bdy",
             "acceleration", "fpn 0.5"]
    if rain is not None:
        with open(os.path.join(d, "r.txt"), "w") as fh:
            fh.write(rain)
        lines.append(f"rainfile {d}/r.txt")
    with open(os.path.join(d, "c.par"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return os.path.join(d, "c.par")


def test_short_side_form_stays_closed(tmp_path):
    """`N FREE` reads one field, so the reference leaves the side CLOSED."""
    par = _minimal(tmp_path, "N FREE\nS 0 2 FREE\nE 1 FREE\n# W 0 1 FREE\n")
    case, _ = load_par(par)
    assert (case.west_free, case.east_free, case.north_free, case.south_free) == (
        False, False, False, True)
    if orc.ref_available():
        assert orc.RefSim(par).free == (False, False, False, True)


def test_unknown_keys_and_defaults(tmp_path):
    """README spellings (fpn, acceleration) are ignored; parser defaults apply."""
    case, _ = load_par(_minimal(tmp_path, ""))
    assert case.fpn == 0.035 and case.depth_thresh == 0.001 and case.sim_time == 3600.0
    assert case.cfl == 0.7 and case.init_tstep == 10.0 and case.mass_int == 60.0


def test_point_types_and_skips(tmp_path):
    bci = ("P 5 15 QFIX 0.25\n"      # cell (0,0)
           "P 15 5 QVAR hyd\n"       # cell (1,1)
           "P 25 15 HFIX 1.5\n"      # cell (2,0)
           "P 25 5 FREE\n"           # cell (2,1)
           "P 15 15 QVAR\n"          # no name: skipped
           "P 15 15 BOGUS 3\n"       # unknown type: skipped
           "P 5 5 HVAR stage\n")     # cell (0,1)
    bdy = ("title line\nhyd\n2 seconds\n0.5 0\n1.5 100\nstage\n3\n1 0\n2 50\n3 100\n")
    case, f = load_par(_minimal(tmp_path, bci, bdy))
    np.testing.assert_array_equal(f.flow_idx, [0, 4])
    np.testing.assert_array_equal(f.flow_type, [sc.QFIX, sc.QVAR])
    np.testing.assert_array_equal(f.flow_value, [0.25, 0.0])
    np.testing.assert_array_equal(f.flow_times, [0.0, 100.0])
    np.testing.assert_array_equal(f.flow_vals, [0.5, 1.5])
    np.testing.assert_array_equal(f.other_idx, [2, 5, 3])
    np.testing.assert_array_equal(f.other_type, [2, 1, 3])
    np.testing.assert_array_equal(f.other_value, [1.5, 0.0, 0.0])
    np.testing.assert_array_equal(f.other_times, [0.0, 50.0, 100.0])


def test_bdy_first_boundary_with_name_gets_series(tmp_path):
    bci = "P 5 15 QVAR q\nP 15 15 QVAR q\nP 25 15 QVAR q1\n"
    bdy = "t\nq1\n1\n9 0\nq\n1\n7 0\n"
    _, f = load_par(_minimal(tmp_path, bci, bdy))
    np.testing.assert_array_equal(np.diff(f.flow_off), [1, 0, 1])
    np.testing.assert_array_equal(f.flow_vals, [7.0, 9.0])


def test_rain_file(tmp_path):
    _, f = load_par(_minimal(tmp_path, "", rain="header\n1e-6 0\n# c\n2e-6 60\n\n"))
    np.testing.assert_array_equal(f.rain_times, [0.0, 60.0])
    np.testing.assert_array_equal(f.rain_rates, [1e-6, 2e-6])
    d = str(tmp_path / "x")
    os.makedirs(d)
    par = _minimal(tmp_path / "x", "")
    with open(par, "a") as fh:
        fh.write(f"rainfile {d}/missing.txt\n")
    _, f2 = load_par(par)
    assert f2.n_rain == 0  # a missing rain file disables rain, as in the reference


def test_errors(tmp_path):
    with pytest.raises(_lib.AFError) as e:
        load_par(str(tmp_path / "nope.par"))
    assert e.value.code == _lib.AF_EIO
    with pytest.raises(_lib.AFError) as e:
        load_par(_minimal(tmp_path, "P 95 5 QFIX 1\n"))  # x maps to column 9 of 3
    assert e.value.code == _lib.AF_ERANGE
    with pytest.raises(_lib.AFError) as e:
        load_par(_minimal(tmp_path, "", dem_rows=["1 2 3", "4 5"]))  # truncated DEM
    assert e.value.code == _lib.AF_EIO
    with pytest.raises(_lib.AFError) as e:
        load_par(_minimal(tmp_path, "P 5 5 QVAR q\n", "t\nq\nx\n"))  # bad count line
    assert e.value.code == _lib.AF_EIO


def test_large_dem_parsed_in_parallel_equals_sequential_values(tmp_path):
    """Above 1 MB of text the DEM body is converted by several threads; the
    values are the sequential reader's (round-trip text, formats of all kinds)."""
    rng = np.random.default_rng(8)
    ny, nx = 300, 410
    dem = rng.normal(20.0, 5.0, size=(ny, nx))
    dem[::7, ::5] = sc.NODATA
    case = sc.Case(nx, ny, 2.0, dem, name="big")
    par = case.write(str(tmp_path))
    got, _ = load_par(par)
    np.testing.assert_array_equal(got.dem, dem)
    # hand-written text: mixed spacing, exponents, integers, line breaks anywhere
    vals = rng.uniform(-50, 50, size=nx * ny)
    toks = []
    for k, v in enumerate(vals):
        toks.append(("%.17g" if k % 3 else "%.6e") % v)
    text = ("ncols %d\nnrows %d\nxllcorner 0\nyllcorner 0\ncellsize 1\nNODATA_value -9999\n"
            % (nx, ny))
    text += "".join(t + ("\n" if k % 97 == 0 else "  \t " if k % 5 == 0 else " ")
                    for k, t in enumerate(toks))
    path = tmp_path / "mixed.asc"
    path.write_text(text)
    want = np.array([float(t) for t in toks]).reshape(ny, nx)
    case2 = sc.Case(nx, ny, 1.0, np.zeros((ny, nx)), name="mixed")
    par2 = case2.write(str(tmp_path / "mixed_case"))
    body = open(par2).read().replace(
        "DEMfile " + str(tmp_path / "mixed_case" / "dem.asc"), "DEMfile " + str(path))
    open(par2, "w").write(body)
    got2, _ = load_par(par2)
    np.testing.assert_array_equal(got2.dem, want)
    # a malformed token deep in the body and a truncated body are errors
    for bad in (text.replace(toks[nx * ny // 2], toks[nx * ny // 2] + "x", 1),
                text[: len(text) * 3 // 4]):
        path.write_text(bad)
        with pytest.raises(_lib.AFError):
            load_par(par2)


def test_par_outputs_and_stage_points(tmp_path):
    """The output keys of a .par file and its stage points as the reference's
    CLI reads them (src/io.cpp:9-85): '#' comments skipped, world
    coordinates mapped by truncation, a missing name numbered "Stage<n>", a
    point off the grid kept with no cell (NaN in stage.csv)."""
    from adaptflood_b200.sim import par_outputs
    c = sc.small_case(70, 50, seed=51, sim_time=300.0)
    c.xll, c.yll = 1000.0, 2000.5
    par = c.write(str(tmp_path / "in"), out_dir=str(tmp_path / "out"))
    top = c.yll + c.ny * c.dx
    with open(tmp_path / "st.txt", "w") as f:
        f.write("# gauges\n")
        f.write(f"{c.xll + 10.5 * c.dx} {top - 12.5 * c.dx} gauge_a\n")
        f.write(f"{c.xll + 3.5 * c.dx} {top - 2.5 * c.dx}\n")
        f.write(f"{c.xll + 5.5 * c.dx} {c.yll - 30 * c.dx} outside\n")
    with open(par, "a") as f:
        f.write(f"stagefile {tmp_path / 'st.txt'}\nstageint 30\noutput_format 2\nvoutput 1\n"
                "async_output 1\nsaveint 120\n")
    o = par_outputs(par)
    assert o["out_dir"] == str(tmp_path / "out")
    assert (o["save_int"], o["stage_int"], o["output_format"]) == (120.0, 30.0, 2)
    assert o["voutput"] and o["async_style"]
    assert o["stages"] == [("gauge_a", 10 + 12 * c.nx), ("Stage2", 3 + 2 * c.nx), ("outside", -1)]


def test_par_without_stage_file_has_no_stage_points(tmp_path):
    from adaptflood_b200.sim import par_outputs
    c = sc.small_case(20, 10, seed=3, sim_time=60.0)
    par = c.write(str(tmp_path / "in"), out_dir=str(tmp_path / "out"))
    with open(par, "a") as f:
        f.write(f"stagefile {tmp_path / 'missing.txt'}\n")
    o = par_outputs(par)
    assert o["stages"] == [] and o["output_format"] == 0 and not o["async_style"]
