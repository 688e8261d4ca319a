"""Autotuner of the batch layer's tile shapes.

A strip of the fused step is 30*N columns (one warp, N cells per lane) by R
rows; R is the free tile dimension.  Short strips give more warps per grid
(small grids fill the GPU) but pay the strip prologue (one extra row of H,
DEM and Qx, and the recomputed face row) more often; tall strips amortise it
but leave SMs idle on small grids.  The best R depends on the grid size, so
the batch keeps one R per size class (floor(log2(cells))).

``tune_rows`` measures, for each size class asked for, a batch of wet
synthetic grids of that class large enough to fill the GPU, at each candidate
R, and returns the fastest R per class (cell-updates/s, CUDA events on the
batch's stream, after warm-up steps; the better of two timings).  The
load-adaptive strip height is off while it measures, so each candidate runs
at its own height (with it on, the taller candidates would be cut down to the
same height and the choice among them would be noise); a batch that uses
the tuned heights keeps it on, to lower them when few scenarios remain.  ``tune_variant`` picks the launch
shape (warps per block x resident blocks per SM) of the batch kernel the
same way.  Results do not depend on R or the variant (bit for bit), only
the speed does.
"""
from __future__ import annotations

import math
from typing import Dict, Iterable, Optional, Sequence

import numpy as np

from . import scenarios as sc
from .batch import Batch

ROWS = (2, 4, 8, 16, 32, 64)
VARIANTS = (0, 1, 2, 3, 4)


def _probe_case(cls: int, seed: int = 0) -> sc.Case:
    """A wet grid of size class `cls` (2^cls <= cells < 2^(cls+1)), aspect 1:2,
    every face active (a film on a gently sloped plane with ripples)."""
    cells = int(2 ** (cls + 0.5))
    nx = max(8, int(round(math.sqrt(cells / 2.0))))
    ny = max(8, cells // nx)
    while nx * ny >= 2 ** (cls + 1):
        ny -= 1
    while nx * ny < 2 ** cls:
        ny += 1
    dx = 5.0
    j = np.arange(ny, dtype=np.float64)[:, None]
    i = np.arange(nx, dtype=np.float64)[None, :]
    dem = 0.001 * dx * (ny - 1 - j) + 0.2 * np.sin(i / 7.0 + seed) * np.cos(j / 5.0)
    c = sc.Case(nx, ny, dx, dem, sim_time=1e9, save_int=1e9, mass_int=60.0, west_free=True,
                east_free=True, north_free=True, south_free=True, name=f"probe_{cls}")
    c.h0 = np.full((ny, nx), 0.05)
    return c


def _rate(batch: Batch, cases: Sequence[sc.Case], steps: int, warmup: int,
          repeats: int = 2) -> float:
    import torch
    slots = [batch.add(c) for c in cases]
    batch.run(max_steps=warmup)
    stream = torch.cuda.ExternalStream(batch.stream)
    ms = float("inf")
    for _ in range(repeats):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.launch(max_steps=steps)
        e1.record(stream)
        batch.sync()
        ms = min(ms, e0.elapsed_time(e1))
    for s in slots:
        batch.remove(s)
    return sum(c.cells for c in cases) * steps / (ms / 1e3)


def _fill(cls: int, target_cells: int, cap: int = 256):
    one = _probe_case(cls)
    count = max(1, min(cap, target_cells // one.cells))
    return [one] * count


def tune_rows(classes: Iterable[int], precision: str = "f32", device: int = 0,
              rows: Sequence[int] = ROWS, target_cells: int = 1 << 26, steps: int = 20,
              warmup: int = 3, variant: int = -1, arena_bytes: Optional[int] = None,
              scores_out: Optional[dict] = None) -> Dict[int, int]:
    """The fastest strip height per size class (`scores_out`, if given,
    receives the measured cell-updates/s per class and height)."""
    best: Dict[int, int] = {}
    with Batch(precision, device=device, variant=variant, arena_bytes=arena_bytes) as b:
        b.set_balance(0)
        for cls in classes:
            cases = _fill(cls, target_cells)
            ny = cases[0].ny
            scores = {}
            for r in rows:
                if r > ny and scores:
                    continue
                b.set_rows(cls, r)
                scores[r] = _rate(b, cases, steps, warmup)
            best[cls] = max(scores, key=scores.get)
            if scores_out is not None:
                scores_out[cls] = scores
            b.set_rows(cls, best[cls])
    return best


def tune_variant(classes: Iterable[int], rows: Dict[int, int], precision: str = "f32",
                 device: int = 0, variants: Sequence[int] = VARIANTS,
                 target_cells: int = 1 << 25, steps: int = 12, warmup: int = 3,
                 arena_bytes: Optional[int] = None) -> int:
    """The fastest launch variant of the batch kernel on a mix of the classes."""
    classes = list(classes)
    per = max(1, target_cells // max(1, len(classes)))
    cases = [c for cls in classes for c in _fill(cls, per)]
    scores = {}
    for v in variants:
        with Batch(precision, device=device, variant=v, arena_bytes=arena_bytes) as b:
            for cls, r in rows.items():
                b.set_rows(cls, r)
            scores[v] = _rate(b, cases, steps, warmup)
    return max(scores, key=scores.get)
