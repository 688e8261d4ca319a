"""Seeded synthetic flood cases and their AdaptFlood input files.

A :class:`Case` holds one grid (DEM, optional initial depth), the run
parameters of a ``.par`` file, the line boundaries, the point boundaries with
their hydrographs, and an optional uniform rain series.  ``Case.write()`` emits
the five input files in the formats the reference parses
(src/io.cpp:9-47 ``.par``, :132-161 DEM, :164-254 ``.bci``, :257-296 ``.bdy``,
:103-129 rain), so the same case can be run by the reference and by this
library.

Format facts the writers respect (they are properties of the reference's
parsers, kept here on purpose):

* ``.par`` keys are the parser's spellings (``fpfric``, ``depth_thresh``,
  ``initial_tstep``, ``dirroot``); unknown keys are ignored by the reference.
* A line boundary is only FREE when written ``<side> <a> <b> FREE``: the
  parser's short form ``<side> FREE`` reads one field and leaves the side
  CLOSED (src/io.cpp:224-244).
* Point coordinates are world coordinates mapped with truncation,
  ``x = (int)((X - xll)/cs)``, ``y = (int)((yll + nrows*cs - Y)/cs)``
  (src/io.cpp:185-187); writers use cell centres.
* ``.bdy`` series lines are ``value time`` (src/io.cpp:281-284).
* Discharges (QFIX/QVAR) are per unit width, m^2/s; m^3/s = value * dx.
* HFIX/HVAR values are depths (H = value, src/kernels.cpp:270-273).
* Rain rates are m/s; a piecewise-constant series is written as two points
  per interval with repeated boundary times (the reader interpolates
  linearly, and a zero-length segment never matches, src/io.cpp:93-98).

The configurations are those of the benchmark definition: C1 512^2 at 10 m
with a 20 m^3/s centre source, C2 8192^2 at 5 m with 4096 QVAR sources, rain
and an HVAR edge point, C3 16384^2 at 2 m with ponds and a reservoir block,
C4 ensembles of 256^2..2048^2 grids, C5 served request streams.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence

import numpy as np

# BoundaryType of src/types.hpp:41-48
CLOSED, FREE, HFIX, HVAR, QFIX, QVAR = 0, 1, 2, 3, 4, 5
_TYPE_NAME = {FREE: "FREE", HFIX: "HFIX", HVAR: "HVAR", QFIX: "QFIX", QVAR: "QVAR"}

NODATA = -9999.0


@dataclasses.dataclass
class PointBC:
    """One ``P`` line of a ``.bci`` file (cell indices, not world coords)."""

    kind: int
    i: int
    j: int
    value: float = 0.0
    name: str = ""
    times: Optional[np.ndarray] = None
    values: Optional[np.ndarray] = None


@dataclasses.dataclass
class Case:
    nx: int
    ny: int
    dx: float
    dem: np.ndarray  # float64 [ny, nx], row 0 = north
    xll: float = 0.0
    yll: float = 0.0
    nodata: float = NODATA
    h0: Optional[np.ndarray] = None  # initial depth, float64 [ny, nx]
    sim_time: float = 3600.0
    save_int: float = 600.0
    mass_int: float = 60.0
    init_tstep: float = 10.0
    cfl: float = 0.7
    fpn: float = 0.035
    depth_thresh: float = 0.001
    west_free: bool = False
    east_free: bool = False
    north_free: bool = False
    south_free: bool = False
    points: List[PointBC] = dataclasses.field(default_factory=list)
    rain_times: Optional[np.ndarray] = None
    rain_rates: Optional[np.ndarray] = None
    name: str = "case"

    # ------------------------------------------------------------------ sizes
    @property
    def cells(self) -> int:
        return self.nx * self.ny

    def flow_points(self) -> List[PointBC]:
        return [p for p in self.points if p.kind in (QFIX, QVAR)]

    def other_points(self) -> List[PointBC]:
        return [p for p in self.points if p.kind in (FREE, HFIX, HVAR)]

    # ------------------------------------------------------------ file output
    def write(self, directory: str, out_dir: Optional[str] = None) -> str:
        """Write ``case.par`` and its input files; returns the ``.par`` path.

        Paths inside the ``.par`` file are absolute, because the reference
        opens them relative to the working directory.
        """
        directory = os.path.abspath(directory)
        os.makedirs(directory, exist_ok=True)
        dem_path = os.path.join(directory, "dem.asc")
        bci_path = os.path.join(directory, "case.bci")
        bdy_path = os.path.join(directory, "case.bdy")
        rain_path = os.path.join(directory, "case.rain")
        par_path = os.path.join(directory, "case.par")
        out_dir = out_dir or os.path.join(directory, "results")
        write_dem(dem_path, self.dem, self.xll, self.yll, self.dx, self.nodata)
        with open(bci_path, "w") as f:
            f.write("# generated case\n")
            last_row = self.ny - 1
            last_col = self.nx - 1
            if self.north_free:
                f.write(f"N 0 {last_col} FREE\n")
            if self.south_free:
                f.write(f"S 0 {last_col} FREE\n")
            if self.east_free:
                f.write(f"E 0 {last_row} FREE\n")
            if self.west_free:
                f.write(f"W 0 {last_row} FREE\n")
            for p in self.points:
                X = self.xll + (p.i + 0.5) * self.dx
                Y = self.yll + self.ny * self.dx - (p.j + 0.5) * self.dx
                tail = ""
                if p.kind in (QFIX, HFIX):
                    tail = " " + repr(float(p.value))
                elif p.kind in (QVAR, HVAR):
                    tail = " " + p.name
                f.write(f"P {X!r} {Y!r} {_TYPE_NAME[p.kind]}{tail}\n")
        with open(bdy_path, "w") as f:
            f.write("generated boundary series\n")
            for p in self.points:
                if p.kind not in (QVAR, HVAR) or p.times is None:
                    continue
                f.write(f"{p.name}\n{len(p.times)} seconds\n")
                for v, t in zip(p.values, p.times):
                    f.write(f"{float(v)!r} {float(t)!r}\n")
        lines = [
            f"DEMfile {dem_path}",
            f"bcifile {bci_path}",
            f"bdyfile {bdy_path}",
            f"dirroot {out_dir}",
            f"sim_time {self.sim_time!r}",
            f"saveint {self.save_int!r}",
            f"massint {self.mass_int!r}",
            f"initial_tstep {self.init_tstep!r}",
            f"cfl {self.cfl!r}",
            f"fpfric {self.fpn!r}",
            f"depth_thresh {self.depth_thresh!r}",
            "async_output 0",
        ]
        if self.rain_times is not None and len(self.rain_times):
            with open(rain_path, "w") as f:
                f.write("rate(m/s) time(s)\n")
                for r, t in zip(self.rain_rates, self.rain_times):
                    f.write(f"{float(r)!r} {float(t)!r}\n")
            lines.append(f"rainfile {rain_path}")
        with open(par_path, "w") as f:
            f.write("# generated AdaptFlood case\n")
            f.write("\n".join(lines) + "\n")
        return par_path


def write_dem(path: str, dem: np.ndarray, xll: float, yll: float, cs: float,
              nodata: float) -> None:
    """ESRI ASCII grid with round-trip (17 significant digit) values."""
    ny, nx = dem.shape
    with open(path, "w") as f:
        f.write(f"ncols {nx}\nnrows {ny}\nxllcorner {xll!r}\nyllcorner {yll!r}\n"
                f"cellsize {cs!r}\nNODATA_value {nodata!r}\n")
        for j in range(ny):
            f.write(" ".join(repr(float(v)) for v in dem[j]))
            f.write("\n")


# ---------------------------------------------------------------- terrain
def _value_noise_rows(lat: np.ndarray, spacing: float, j0: int, j1: int, nx: int,
                      x0: int = 0) -> np.ndarray:
    """Smooth value noise in [-1, 1] for rows j0..j1, columns x0..x0+nx, from a
    random lattice."""
    y = (np.arange(j0, j1, dtype=np.float64) + 0.5) / spacing
    x = (np.arange(x0, x0 + nx, dtype=np.float64) + 0.5) / spacing
    iy = np.floor(y).astype(np.int64)
    ix = np.floor(x).astype(np.int64)
    fy = y - iy
    fx = x - ix
    sy = fy * fy * (3.0 - 2.0 * fy)
    sx = fx * fx * (3.0 - 2.0 * fx)
    a = lat[iy][:, ix]
    b = lat[iy][:, ix + 1]
    c = lat[iy + 1][:, ix]
    d = lat[iy + 1][:, ix + 1]
    top = a + (b - a) * sx[None, :]
    bot = c + (d - c) * sx[None, :]
    return 2.0 * (top + (bot - top) * sy[:, None]) - 1.0


def make_dem(nx: int, ny: int, dx: float, seed: int, slope: float = 0.001,
             amplitude: float = 0.5, channel_depth: float = 3.0, channel_width: int = 5,
             ponds: int = 0, pond_depth=(0.5, 2.0), rows_per_chunk: int = 512,
             window=None) -> np.ndarray:
    """Plane sloping ``slope`` toward the south + 2-octave seeded noise of
    amplitude ``amplitude`` (a product of sinusoids plus two octaves of value
    noise) + an N-S channel ``channel_width`` cells wide, ``channel_depth``
    deep, centred on column nx//2; optional Gaussian ponds.

    ``window`` = (x0, y0, w, h) returns only that window of the nx x ny DEM,
    computed cell by cell with the same expressions (the same values as a
    crop of the whole DEM, without building it)."""
    x0, y0, wx, wy = window if window is not None else (0, 0, nx, ny)
    if not (0 <= x0 and 0 <= y0 and x0 + wx <= nx and y0 + wy <= ny):
        raise ValueError("window outside the grid")
    rng = np.random.default_rng(seed)
    s1 = max(4.0, min(nx, ny) / 8.0)
    s2 = s1 / 2.0
    lat1 = rng.random((int(ny / s1) + 3, int(nx / s1) + 3))
    lat2 = rng.random((int(ny / s2) + 3, int(nx / s2) + 3))
    lx = rng.uniform(0.15, 0.35) * nx
    ly = rng.uniform(0.15, 0.35) * ny
    px, py = rng.uniform(0, 2 * math.pi, size=2)
    dem = np.empty((wy, wx), dtype=np.float64)
    xs = np.arange(x0, x0 + wx, dtype=np.float64)
    sinx = np.sin(2 * math.pi * xs / lx + px)
    c0 = max(0, nx // 2 - channel_width // 2)
    c1 = min(nx, c0 + channel_width)
    c0w, c1w = max(c0, x0) - x0, min(c1, x0 + wx) - x0  # the channel inside the window
    for j0 in range(y0, y0 + wy, rows_per_chunk):
        j1 = min(y0 + wy, j0 + rows_per_chunk)
        ys = np.arange(j0, j1, dtype=np.float64)
        siny = np.sin(2 * math.pi * ys / ly + py)
        n = 0.5 * (siny[:, None] * sinx[None, :])
        n += 0.3 * _value_noise_rows(lat1, s1, j0, j1, wx, x0)
        n += 0.2 * _value_noise_rows(lat2, s2, j0, j1, wx, x0)
        z = slope * (ny - 1 - ys)[:, None] * dx + amplitude * n
        if channel_depth and c1w > c0w:
            z[:, c0w:c1w] -= channel_depth
        dem[j0 - y0:j1 - y0] = z
    for _ in range(ponds):
        ci, cj = rng.uniform(0, nx), rng.uniform(0, ny)
        r = rng.uniform(0.004, 0.02) * min(nx, ny) + 2.0
        depth = rng.uniform(*pond_depth)
        i0, i1 = int(max(0, ci - 3 * r)), int(min(nx, ci + 3 * r + 1))
        j0, j1 = int(max(0, cj - 3 * r)), int(min(ny, cj + 3 * r + 1))
        i0, i1 = max(i0, x0), min(i1, x0 + wx)
        j0, j1 = max(j0, y0), min(j1, y0 + wy)
        if i1 <= i0 or j1 <= j0:
            continue
        gi = np.arange(i0, i1) + 0.5 - ci
        gj = np.arange(j0, j1) + 0.5 - cj
        dem[j0 - y0:j1 - y0, i0 - x0:i1 - x0] -= depth * np.exp(
            -(gj[:, None] ** 2 + gi[None, :] ** 2) / (2 * r * r))
    return dem


def triangular_hydrograph(peak: float, rise: float, t0: float, n: int = 30):
    """``n`` entries: 0 at t0, ``peak`` at t0+rise, back to 0 at t0+3*rise."""
    n_up = n // 3
    t_up = np.linspace(t0, t0 + rise, n_up, endpoint=False)
    t_dn = np.linspace(t0 + rise, t0 + 3.0 * rise, n - n_up)
    times = np.concatenate([t_up, t_dn])
    vals = np.where(times <= t0 + rise, peak * (times - t0) / rise,
                    peak * (t0 + 3.0 * rise - times) / (2.0 * rise))
    return times, np.maximum(vals, 0.0)


def piecewise_rain(rng: np.random.Generator, sim_time: float, interval: float = 60.0,
                   max_mm_h: float = 50.0):
    """Piecewise-constant rain (m/s), two points per interval."""
    k = int(math.ceil(sim_time / interval))
    rates = rng.uniform(0.0, max_mm_h, size=k) / 3.6e6
    times = np.empty(2 * k)
    vals = np.empty(2 * k)
    times[0::2] = np.arange(k) * interval
    times[1::2] = (np.arange(k) + 1) * interval
    vals[0::2] = rates
    vals[1::2] = rates
    return times, vals


def wet_prone_cells(dem: np.ndarray, rng: np.random.Generator, count: int,
                    window: int = 4) -> List[tuple]:
    """``count`` distinct cells whose elevation is below their local mean."""
    ny, nx = dem.shape
    chosen, seen = [], set()
    while len(chosen) < count:
        cand = rng.integers(0, nx * ny, size=4 * count)
        for c in cand:
            c = int(c)
            if c in seen:
                continue
            seen.add(c)
            j, i = divmod(c, nx)
            win = dem[max(0, j - window):j + window + 1, max(0, i - window):i + window + 1]
            if dem[j, i] < win.mean():
                chosen.append((i, j))
                if len(chosen) == count:
                    break
        if len(seen) >= nx * ny:
            break
    return chosen


# ------------------------------------------------------------ configurations
def config1(seed: int = 1) -> Case:
    """512x512 at 10 m, one 20 m^3/s QFIX source at the centre, all edges FREE."""
    nx = ny = 512
    dx = 10.0
    dem = make_dem(nx, ny, dx, seed)
    c = Case(nx, ny, dx, dem, sim_time=3600.0, save_int=600.0, mass_int=60.0, cfl=0.7,
             fpn=0.035, depth_thresh=0.001, west_free=True, east_free=True, north_free=True,
             south_free=True, name="c1_512")
    c.points.append(PointBC(QFIX, nx // 2, ny // 2, value=20.0 / dx))
    return c


def config2(seed: int = 2, n: int = 8192, dx: float = 5.0, sources: int = 4096) -> Case:
    """8192x8192 at 5 m: 4096 QVAR triangular hydrographs at wet-prone cells,
    piecewise rain 0-50 mm/h, an HVAR depth 1+sin(2 pi t/7200) on the west
    edge, FREE north/south/east, 7200 s."""
    rng = np.random.default_rng(seed)
    dem = make_dem(n, n, dx, seed)
    c = Case(n, n, dx, dem, sim_time=7200.0, save_int=1800.0, mass_int=60.0, cfl=0.7,
             fpn=0.035, depth_thresh=0.001, east_free=True, north_free=True, south_free=True,
             name=f"c2_{n}")
    for k, (i, j) in enumerate(wet_prone_cells(dem, rng, sources)):
        peak = rng.uniform(0.5, 5.0)
        rise = rng.uniform(300.0, 1200.0)
        t0 = rng.uniform(0.0, 1800.0)
        tt, vv = triangular_hydrograph(peak / dx, rise, t0)
        c.points.append(PointBC(QVAR, i, j, name=f"q{k:05d}", times=tt, values=vv))
    ht = np.linspace(0.0, 7200.0, 31)
    hv = 1.0 + np.sin(2 * math.pi * ht / 7200.0)
    c.points.append(PointBC(HVAR, 0, n // 2, name="stage_w", times=ht, values=hv))
    c.rain_times, c.rain_rates = piecewise_rain(rng, c.sim_time)
    return c


def config3(seed: int = 3, n: int = 16384, dx: float = 2.0, block: int = 512,
            channel: bool = True) -> Case:
    """16384x16384 at 2 m with Gaussian ponds and a 1 m deep reservoir block.
    At full size the reservoir (at n/4) is 8 km from the DEM's 3 m deep
    channel (at n/2), which its water does not reach in the 3 h simulated;
    reduced grids that keep the reservoir should drop the channel
    (channel=False): deep water in it in a closed box is outside the stable
    regime of the scheme."""
    dem = make_dem(n, n, dx, seed, ponds=max(8, (n // 256) ** 2 // 4),
                   channel_depth=3.0 if channel else 0.0)
    h0 = np.zeros((n, n), dtype=np.float64)
    b0 = n // 4
    h0[b0:b0 + block, b0:b0 + block] = 1.0
    return Case(n, n, dx, dem, h0=h0, sim_time=10800.0, save_int=3600.0, mass_int=600.0,
                cfl=0.7, fpn=0.035, depth_thresh=0.001, name=f"c3_{n}")


def config3_window(w: int = 1024, seed: int = 3, n: int = 16384, dx: float = 2.0,
                   block: int = 512) -> Case:
    """A w x w window of the C3 configuration centred on its reservoir: the
    same terrain, ponds and 1 m deep reservoir block cell for cell (closed
    edges at the window), without building the full grid."""
    b0 = n // 4
    x0 = y0 = max(0, b0 + block // 2 - w // 2)
    dem = make_dem(n, n, dx, seed, ponds=max(8, (n // 256) ** 2 // 4), window=(x0, y0, w, w))
    h0 = np.zeros((w, w), dtype=np.float64)
    r0 = b0 - y0
    h0[max(0, r0):r0 + block, max(0, r0):r0 + block] = 1.0
    return Case(w, w, dx, dem, h0=h0, sim_time=10800.0, save_int=3600.0, mass_int=600.0,
                cfl=0.7, fpn=0.035, depth_thresh=0.001, name=f"c3_window_{w}")


def ensemble_case(rng: np.random.Generator, seed: int, lo: int = 256, hi: int = 2048,
                  sim_time: float = 1800.0) -> Case:
    """One member of an ensemble: log-uniform cell count in [lo^2, hi^2],
    aspect 1:1..1:4, Manning n U(0.02, 0.08), 1-64 QFIX/QVAR sources."""
    cells = math.exp(rng.uniform(math.log(lo * lo), math.log(hi * hi)))
    aspect = rng.uniform(1.0, 4.0)
    nx = max(16, int(round(math.sqrt(cells * aspect))))
    ny = max(16, int(round(cells / nx)))
    if rng.random() < 0.5:
        nx, ny = ny, nx
    dx = float(rng.choice([2.0, 5.0, 10.0]))
    dem = make_dem(nx, ny, dx, seed)
    c = Case(nx, ny, dx, dem, sim_time=sim_time, save_int=sim_time, mass_int=60.0, cfl=0.7,
             fpn=float(rng.uniform(0.02, 0.08)), depth_thresh=0.001, west_free=True,
             east_free=True, north_free=True, south_free=True, name=f"ens_{seed}")
    ns = int(rng.integers(1, 65))
    for k, (i, j) in enumerate(wet_prone_cells(dem, rng, ns)):
        if rng.random() < 0.5:
            c.points.append(PointBC(QFIX, i, j, value=float(rng.uniform(0.5, 5.0)) / dx))
        else:
            tt, vv = triangular_hydrograph(float(rng.uniform(0.5, 5.0)) / dx,
                                           float(rng.uniform(300.0, 1200.0)),
                                           float(rng.uniform(0.0, sim_time / 2)))
            c.points.append(PointBC(QVAR, i, j, name=f"q{k:03d}", times=tt, values=vv))
    return c


def config4(seed: int = 4, count: int = 256, lo: int = 256, hi: int = 2048,
            sim_time: float = 1800.0) -> List[Case]:
    rng = np.random.default_rng(seed)
    return [ensemble_case(rng, seed * 100003 + k, lo, hi, sim_time) for k in range(count)]


def config5(seed: int = 5, count: int = 32, lo: int = 128, hi: int = 4096,
            sim_time=(600.0, 3600.0)) -> List[Case]:
    """Served-loop requests: grids log-uniform in [lo^2, hi^2] cells with the
    ensemble generator, each with its own sim_time drawn from U(sim_time)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        st = float(rng.uniform(*sim_time))
        out.append(ensemble_case(rng, seed * 100019 + k, lo, hi, sim_time=st))
    return out


def small_case(nx: int, ny: int, seed: int, dx: float = 10.0, free: Sequence[bool] = (1, 1, 1, 1),
               n_qfix: int = 1, n_qvar: int = 1, n_hfix: int = 0, n_hvar: int = 0,
               n_free_pts: int = 0, dup_sources: bool = False, rain: bool = False,
               nodata_block: bool = False, h0: bool = False, sim_time: float = 600.0,
               channel: bool = True) -> Case:
    """A small case with every feature switchable (parity tests)."""
    rng = np.random.default_rng(seed)
    dem = make_dem(nx, ny, dx, seed, channel_depth=3.0 if channel else 0.0,
                   channel_width=min(5, max(1, nx // 8)))
    if nodata_block and nx >= 8 and ny >= 8:
        dem[ny // 4: ny // 4 + 3, nx // 5: nx // 5 + 4] = NODATA
        dem[ny - 1, nx - 3:] = NODATA
    c = Case(nx, ny, dx, dem, sim_time=sim_time, save_int=sim_time / 2, mass_int=60.0,
             cfl=0.7, fpn=0.035, depth_thresh=0.001, west_free=bool(free[0]),
             east_free=bool(free[1]), north_free=bool(free[2]), south_free=bool(free[3]),
             name=f"small_{nx}x{ny}_{seed}")
    cells = [(int(rng.integers(0, nx)), int(rng.integers(0, ny))) for _ in range(64)]
    k = 0
    for _ in range(n_qfix):
        i, j = cells[k % len(cells)]; k += 1
        c.points.append(PointBC(QFIX, i, j, value=float(rng.uniform(0.2, 2.0))))
    for q in range(n_qvar):
        i, j = cells[k % len(cells)]; k += 1
        tt, vv = triangular_hydrograph(float(rng.uniform(0.2, 2.0)), float(rng.uniform(30, 120)),
                                       float(rng.uniform(0, 60)))
        c.points.append(PointBC(QVAR, i, j, name=f"qv{q}", times=tt, values=vv))
    if dup_sources and c.points:
        first = c.points[0]
        c.points.append(PointBC(QFIX, first.i, first.j, value=0.75))
        tt, vv = triangular_hydrograph(0.9, 40.0, 10.0)
        c.points.append(PointBC(QVAR, first.i, first.j, name="qdup", times=tt, values=vv))
    for _ in range(n_hfix):
        i, j = cells[k % len(cells)]; k += 1
        c.points.append(PointBC(HFIX, i, j, value=float(rng.uniform(0.1, 1.5))))
    for h in range(n_hvar):
        i, j = cells[k % len(cells)]; k += 1
        tt = np.linspace(0.0, sim_time, 13)
        vv = 0.5 + 0.4 * np.sin(2 * math.pi * tt / sim_time)
        c.points.append(PointBC(HVAR, i, j, name=f"hv{h}", times=tt, values=vv))
    for _ in range(n_free_pts):
        i, j = cells[k % len(cells)]; k += 1
        c.points.append(PointBC(FREE, i, j))
    if rain:
        c.rain_times, c.rain_rates = piecewise_rain(rng, sim_time, interval=30.0, max_mm_h=80.0)
    if h0:
        c.h0 = np.zeros((ny, nx))
        c.h0[ny // 3: ny // 3 + max(1, ny // 6), nx // 3: nx // 3 + max(1, nx // 6)] = 0.8
    return c


def wet_start(case: Case, film: float = 0.025, channel_fill: float = 2.0,
              channel_width: int = 5) -> np.ndarray:
    """A seeded-free, deterministic flooded state for throughput runs: a
    ``film`` of water on every valid cell (rain accumulated so far) and the
    N-S channel filled to ``channel_fill`` m, so every face is wet and the
    whole step path (friction pow, sqrt, divisions) runs on every cell."""
    h = np.where(case.dem != case.nodata, film, 0.0)
    c0 = max(0, case.nx // 2 - channel_width // 2)
    h[:, c0:c0 + channel_width] = channel_fill
    return h
