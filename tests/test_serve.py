"""The serving loop's scheduling on the host, driven by a stand-in batch (no
device): every request completes with the right step count, admission never
exceeds the arena, an oversized request is refused, requests that arrive
while a launch runs are admitted and raise the attention flag, and the loop
keeps the batch's rules (no read-back of a running scenario during a launch,
no launch while one is in flight)."""
import math

import numpy as np

from adaptflood_b200 import scenarios as sc
from adaptflood_b200.batch import Arena
from adaptflood_b200.serve import Request, Server, poisson_arrivals, summary


class FakeBatch:
    """Batch's interface on the host: each scenario advances by a fixed dt
    per batch step; a launch completes after a few polls."""

    def __init__(self, arena_bytes, dt=7.0, polls=3):
        self.arena_bytes = arena_bytes
        self.plan = Arena(arena_bytes)
        self.dt = dt
        self.polls = polls
        self.slots = {}
        self.in_flight = False
        self.launch_args = None
        self.attn = False
        self.attn_count = 0
        self.peak_used = 0
        self.next_slot = 0
        self.deferred = []

    def footprint(self, case, forcing=None, t_stop=None):
        return case.cells * 28

    def try_add(self, case, forcing=None, t_stop=None):
        off = self.plan.alloc(self.footprint(case))
        if off is None:
            return None
        s = self.next_slot
        self.next_slot += 1
        self.slots[s] = dict(case=case, stop=t_stop, t=0.0, steps=0, off=off)
        self.peak_used = max(self.peak_used, self.plan.stats()[0])
        return s

    def _finished(self, s):
        d = self.slots[s]
        return not d["t"] < d["stop"]

    def launch(self, max_steps=1 << 40, stop_on_done=False):
        assert not self.in_flight, "launch while a launch is in flight"
        self.in_flight = True
        self.launch_args = (max_steps, stop_on_done)
        self.attn = False
        self.left = self.polls

    def attention(self):
        self.attn = True
        self.attn_count += 1

    def done(self):
        self.left -= 1
        return self.left <= 0

    def sync(self):
        assert self.in_flight
        max_steps, stop_on_done = self.launch_args
        for _ in range(max_steps):
            act = [s for s in self.slots if not self._finished(s)]
            if not act:
                break
            for s in act:
                self.slots[s]["t"] += self.dt
                self.slots[s]["steps"] += 1
            if self.attn or (stop_on_done and any(self._finished(s) for s in act)):
                break
        self.in_flight = False
        for s in self.deferred:
            self.plan.free(self.slots.pop(s)["off"])
        self.deferred.clear()

    def status(self, s):
        d = self.slots[s]
        return d["t"], self.dt, 0.0, d["steps"], 1 if self._finished(s) else 0

    def depth(self, s):
        assert self._finished(s) or not self.in_flight, "read-back of a running scenario"
        c = self.slots[s]["case"]
        return np.full((c.ny, c.nx), float(self.slots[s]["steps"]))

    def remove(self, s):
        if self.in_flight:
            self.deferred.append(s)
        else:
            self.plan.free(self.slots.pop(s)["off"])

    def close(self):
        pass


def _requests(n, rate, seed=0):
    rng = np.random.default_rng(seed)
    arr = poisson_arrivals(rate, n, rng)
    out = []
    for k in range(n):
        nx, ny = int(rng.integers(8, 64)), int(rng.integers(8, 64))
        c = sc.Case(nx, ny, 10.0, np.zeros((ny, nx)), sim_time=float(rng.uniform(30, 400)))
        out.append(Request(k, float(arr[k]), c))
    return out


def test_all_requests_complete_with_their_own_step_counts():
    reqs = _requests(40, rate=2000.0)
    fb = FakeBatch(arena_bytes=1 << 30)
    with Server(batch=fb) as srv:
        srv.run(reqs, poll_s=1e-5)
    for r in reqs:
        assert r.error is None
        assert r.steps == math.ceil(r.stop / fb.dt), (r.rid, r.steps)
        assert r.result is not None and r.result[0, 0] == r.steps
        assert r.completed >= r.admitted >= r.arrival - 1e-9
    s = summary(reqs)
    assert s["requests"] == 40 and s["failed"] == 0
    assert s["p99_latency_s"] >= s["p50_latency_s"] > 0


def test_admission_respects_the_arena_and_refuses_oversized_requests():
    reqs = _requests(30, rate=5000.0, seed=1)
    big = sc.Case(200, 200, 10.0, np.zeros((200, 200)), sim_time=50.0)
    reqs.append(Request(99, 0.0, big))
    cap = 3 * 64 * 64 * 28  # at most three of the largest requests at once
    fb = FakeBatch(arena_bytes=cap)
    with Server(batch=fb) as srv:
        srv.run(reqs, poll_s=1e-5)
    assert fb.peak_used <= cap
    assert reqs[-1].error is not None  # larger than the whole arena
    for r in reqs[:-1]:
        assert r.error is None and r.steps == math.ceil(r.stop / fb.dt)


def test_late_arrivals_raise_attention():
    reqs = _requests(12, rate=200.0, seed=2)
    for r in reqs:
        r.case.sim_time = 5000.0  # long enough that launches are still running
    fb = FakeBatch(arena_bytes=1 << 30, dt=50.0, polls=400)
    with Server(batch=fb) as srv:
        srv.run(reqs, poll_s=2e-4)
    assert fb.attn_count >= 1
    assert all(r.steps == 100 for r in reqs)
