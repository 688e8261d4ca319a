"""GPU test of continuous-batching serving: requests arrive while others run,
are admitted by device-memory footprint into a deliberately small arena, and
each result equals the same scenario run alone by the single-grid FP32 path
(bit for bit, so well inside the stated 1e-3 m FP32 depth tolerance)."""
import numpy as np
import pytest

from adaptflood_b200 import scenarios as sc
from adaptflood_b200.batch import Batch
from adaptflood_b200.serve import Request, Server, poisson_arrivals, summary
from adaptflood_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def test_served_results_equal_results_alone(cuda):
    rng = np.random.default_rng(11)
    arr = poisson_arrivals(40.0, 14, rng)
    reqs = []
    for k in range(14):
        nx, ny = int(rng.integers(20, 160)), int(rng.integers(20, 160))
        case = sc.small_case(nx, ny, seed=200 + k, rain=bool(k % 3 == 0), n_hvar=int(k % 4 == 1),
                             sim_time=float(rng.uniform(120, 480)))
        reqs.append(Request(k, float(arr[k]), case))
    with Batch("f32", arena_bytes=1 << 30) as probe:
        need = sorted(probe.footprint(r.case) for r in reqs)
    arena = sum(need[-3:])  # about three of the largest at a time: requests must wait
    with Server("f32", arena_bytes=arena) as srv:
        srv.run(reqs)
        launches = srv.launches
    assert launches > 1
    assert any(r.admitted > r.arrival + 1e-4 for r in reqs)  # some waited for room
    for r in reqs:
        assert r.error is None
        with Simulation(r.case, "f32") as s:
            n = s.run(r.stop)
            alone = s.depth()
        assert r.steps == n
        np.testing.assert_array_equal(r.result, alone)
    s = summary(reqs)
    assert s["failed"] == 0 and s["p99_latency_s"] >= s["p50_latency_s"]
