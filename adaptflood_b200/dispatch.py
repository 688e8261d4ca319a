"""Multi-GPU ensembles by host dispatch: one process per GPU, whole scenarios
as the units of work, no data-path collective.

A scenario never spans GPUs (the time step needs no exchange between
scenarios), so an ensemble scales by giving each rank a share of the
scenarios.  ``partition`` balances the shares by an estimate of each
scenario's work (cell-updates: cells x sim_time / dx, since the CFL step is
proportional to dx at a given depth), longest first onto the least-loaded
rank.  ``run_ensemble`` runs a rank's share in one batch (in waves when the
share does not fit the batch's arena at once) and gathers every scenario's
outcome on all ranks (``all_gather_object``: gloo or NCCL); a rank whose
share fails still joins the gather, and then every rank raises.
"""
from __future__ import annotations

import heapq
from typing import Callable, Dict, List, Optional, Sequence

from . import forcing as fc
from . import scenarios as sc


def work_estimate(case: sc.Case) -> float:
    """Relative cell-updates of a scenario: cells x sim_time / dx."""
    return case.cells * case.sim_time / case.dx


def partition(work: Sequence[float], world: int) -> List[List[int]]:
    """Indices of `work` split into `world` shares, longest first onto the
    least-loaded share (the LPT rule: at most 4/3 of the optimal makespan)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    shares: List[List[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + float(work[k]), r))
    for s in shares:
        s.sort()
    return shares


def _run_share(cases, mine, rank, batch_factory, forcings) -> Dict[int, dict]:
    """Runs the scenarios `mine` in one batch, in waves: each wave admits what
    fits the batch's arena, runs to completion and frees its slots."""
    out: Dict[int, dict] = {}
    b = batch_factory()
    try:
        pending = list(mine)
        while pending:
            slots, later = {}, []
            for k in pending:
                f = forcings[k] if forcings is not None else None
                s = b.try_add(cases[k], f)
                if s is None:
                    later.append(k)
                else:
                    slots[k] = s
            if not slots:
                raise MemoryError(f"scenario {later[0]} does not fit an empty batch arena")
            b.run()
            for k, s in slots.items():
                t, _, _, steps, state = b.status(s)
                out[k] = {"rank": rank, "steps": int(steps), "t": float(t), "state": int(state)}
                b.remove(s)
            pending = later
    finally:
        b.close()
    return out


def run_ensemble(cases: Sequence[sc.Case], rank: int, world: int, dist=None,
                 batch_factory: Optional[Callable[[], object]] = None,
                 forcings: Optional[Sequence[fc.Forcing]] = None) -> Dict[int, dict]:
    """Runs this rank's share of `cases` to their sim_time and returns every
    scenario's outcome ({index: {"rank", "steps", "t", "state"}}) gathered
    from all ranks.  `dist` is torch.distributed (None: one rank);
    `batch_factory` makes the batch (default: an FP32 Batch on the current
    device).

    Every rank takes part in the gather even when its own share failed (it
    sends an error marker instead of outcomes), and then every rank raises
    the same error: no rank is left waiting in the collective for a peer
    that gave up."""
    shares = partition([work_estimate(c) for c in cases], world)
    mine = shares[rank]
    if batch_factory is None:
        from .batch import Batch
        batch_factory = lambda: Batch("f32")  # noqa: E731
    try:
        out = _run_share(cases, mine, rank, batch_factory, forcings)
        part = {"outcomes": out}
    except Exception as e:  # noqa: BLE001 -- reported to every rank below
        if dist is None or world == 1:
            raise
        out = {}
        part = {"error": f"rank {rank}: {type(e).__name__}: {e}"}
    if dist is None or world == 1:
        return out
    gathered: List[Optional[dict]] = [None] * world
    dist.all_gather_object(gathered, part)
    errors = [g["error"] for g in gathered if g and "error" in g]
    if errors:
        raise RuntimeError("ensemble share failed: " + "; ".join(errors))
    merged: Dict[int, dict] = {}
    for g in gathered:
        merged.update((g or {}).get("outcomes", {}))
    return merged
