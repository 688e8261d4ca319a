"""Continuous-batching flood-forecast serving over the batch layer.

Requests (a scenario and its stop time) arrive over time.  The server keeps
every admitted scenario's state resident in one device arena and steps all
active scenarios together (one persistent kernel per batch step, each
scenario with its own dt).  It runs a loop of launches:

* a request that has arrived is admitted as soon as its device-memory
  footprint fits in the free arena space (first come, first served; a
  smaller request may pass a larger one that does not fit yet);
* requests admitted while a launch is running are uploaded on a separate
  copy stream at once, and the running launch is asked (the attention flag)
  to stop after its current step, so they join within one step;
* a launch also stops when a scenario finishes; the finished scenario's
  depth field is read back while the next launch already runs, then its
  space is released for the requests that wait.

Latency is completion time (result on the host) minus arrival time.  The
same requests can be served one at a time by the single-grid path
(:func:`serve_one_at_a_time`) for comparison.  A scenario's result does not
depend on when it was admitted or on what else ran beside it (bit for bit).
"""
from __future__ import annotations

import collections
import dataclasses
import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import forcing as fc
from . import scenarios as sc
from .batch import FAILED, Batch


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float              # seconds after the start of the run
    case: sc.Case
    forcing: Optional[fc.Forcing] = None
    t_stop: Optional[float] = None
    # filled in by the server
    admitted: float = float("nan")
    completed: float = float("nan")
    steps: int = 0
    result: Optional[np.ndarray] = None
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.completed - self.arrival

    @property
    def stop(self) -> float:
        return self.case.sim_time if self.t_stop is None else self.t_stop


def poisson_arrivals(rate: float, n: int, rng: np.random.Generator) -> np.ndarray:
    """Arrival times (s) of n requests of a Poisson process of `rate` per s."""
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


class Server:
    """Serves requests on one device with one batch."""

    def __init__(self, precision: str = "f32", device: int = 0,
                 arena_bytes: Optional[int] = None, rows: Optional[Dict[int, int]] = None,
                 variant: int = -1, quantum: int = 4096, keep_results: bool = True,
                 clock: Callable[[], float] = time.perf_counter, batch=None):
        # `batch`: an object with Batch's interface to serve with instead
        # (the scheduling tests drive the loop with a host-only stand-in).
        self.batch = batch if batch is not None else Batch(
            precision, device=device, arena_bytes=arena_bytes, variant=variant, rows=rows)
        self.quantum = quantum
        self.keep_results = keep_results
        self.clock = clock
        self.launches = 0

    def close(self) -> None:
        self.batch.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, requests: List[Request], poll_s: float = 50e-6) -> List[Request]:
        """Serves `requests` (arrival times relative to now) to completion."""
        b = self.batch
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting: List[Request] = []
        active: Dict[int, Request] = {}
        finished: List[int] = []
        t0 = self.clock()
        now = lambda: self.clock() - t0  # noqa: E731
        cap = b.arena_bytes

        def arrive():
            while pending and pending[0].arrival <= now():
                r = pending.popleft()
                if b.footprint(r.case, r.forcing, r.stop) > cap:
                    r.error = "footprint larger than the arena"
                    r.completed = now()
                    continue
                waiting.append(r)

        def admit() -> int:
            n = 0
            for r in list(waiting):
                s = b.try_add(r.case, r.forcing, r.stop)
                if s is None:
                    continue
                waiting.remove(r)
                r.admitted = now()
                active[s] = r
                n += 1
            return n

        def collect():
            for s in finished:
                r = active.pop(s)
                r.steps = b.status(s)[3]
                if b.status(s)[4] == FAILED:
                    r.error = "diverged (non-finite or non-positive dt)"
                elif self.keep_results:
                    r.result = b.depth(s)
                else:
                    b.depth(s)  # the readback is part of the latency either way
                b.remove(s)
                r.completed = now()
            finished.clear()

        while pending or waiting or active:
            arrive()
            admit()
            running = any(r is not None and s not in finished for s, r in active.items())
            if running:
                b.launch(max_steps=self.quantum, stop_on_done=True)
                self.launches += 1
            collect()  # overlaps with the launch
            if not running:
                if pending and not waiting:
                    dt = pending[0].arrival - now()
                    if dt > 0:
                        time.sleep(min(dt, 0.01))
                continue
            while not b.done():
                arrive()
                if waiting and admit():
                    b.attention()
                time.sleep(poll_s)
            b.sync()
            for s in list(active):
                if s not in finished and b.status(s)[4] != 0:
                    finished.append(s)
        return requests


def serve_one_at_a_time(requests: List[Request], precision: str = "f64", device: int = 0,
                        keep_results: bool = True,
                        clock: Callable[[], float] = time.perf_counter) -> List[Request]:
    """The plain path: each request in arrival order as its own single-grid
    Simulation (created from host arrays, run to its stop time, depth read
    back), one after another."""
    from .sim import Simulation
    t0 = clock()
    for r in sorted(requests, key=lambda r: r.arrival):
        wait = r.arrival - (clock() - t0)
        if wait > 0:
            time.sleep(wait)
        r.admitted = clock() - t0
        with Simulation(r.case, precision, device=device, forcing=r.forcing) as s:
            r.steps = s.run(r.stop)
            h = s.depth()
        if keep_results:
            r.result = h
        r.completed = clock() - t0
    return requests


def summary(requests: List[Request]) -> dict:
    ok = [r for r in requests if r.error is None]
    lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
    span = max(r.completed for r in requests) - min(r.arrival for r in requests)
    cu = sum(r.case.cells * r.steps for r in ok)
    return {"requests": len(requests), "failed": len(requests) - len(ok),
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()),
            "scenarios_per_s": len(ok) / span if span > 0 else float("nan"),
            "cell_updates_per_s": cu / span if span > 0 else float("nan"),
            "span_s": span}
