"""The serving loop's scheduling on the host, driven by a stand-in batch (no
device): every request completes with the right step count, admission never
exceeds the arena, an oversized request is refused, requests that arrive
while a launch runs are admitted and raise the attention flag, and the loop
keeps the batch's rules (no read-back of a running scenario during a launch,
no launch while one is in flight)."""
import math

import numpy as np

from adaptflood_b200 import scenarios as sc
from adaptflood_b200.serve import Request, Server, poisson_arrivals, summary

from _fakes import FakeBatch


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
