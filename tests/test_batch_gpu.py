"""GPU tests of the batch layer (af_batch_*): many grids of uneven sizes with
their own dt stepped together by one persistent kernel.

Bar: every scenario of a batch ends bit for bit where a single-grid
Simulation of the same case and precision ends (same step count, same H, Qx,
Qy), whatever the other members, the order and time of admission, or the
strip heights; FP64 members are therefore within 1e-9 m of the reference
like the single-grid path.  Volume diagnostics are summed per strip, so they
agree with the single-grid series to 1e-12 relative, not bit for bit.
"""
import numpy as np
import pytest

from adaptflood_b200 import forcing as fc
from adaptflood_b200 import scenarios as sc
from adaptflood_b200.batch import FINISHED, RUNNING, Batch, size_class
from adaptflood_b200.sim import Simulation
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

ARENA = 1 << 30


def _cases():
    """Uneven grids exercising every feature: rain, every edge kind, QFIX/QVAR
    (incl. duplicates on one cell), HFIX/HVAR/FREE points, nodata, an initial
    depth, grids narrower than one strip and taller than many strips."""
    return [
        sc.small_case(131, 77, seed=31, rain=True, n_hvar=1, sim_time=420.0),
        sc.small_case(250, 203, seed=32, free=(1, 0, 1, 1), nodata_block=True, n_hfix=1,
                      dup_sources=True, sim_time=300.0),
        sc.small_case(61, 300, seed=33, free=(0, 1, 0, 1), h0=True, n_free_pts=1, sim_time=360.0),
        sc.small_case(24, 19, seed=34, rain=True, sim_time=500.0),
        sc.small_case(400, 33, seed=35, free=(1, 1, 0, 0), n_qvar=3, sim_time=240.0),
    ]


def _alone(case, prec):
    with Simulation(case, prec) as s:
        n = s.run(case.sim_time)
        t, _, _, steps = s.status()
        st = s.state()
        mass = s.mass_series()
    return n, t, st, mass


def _assert_same(st, ref):
    for k in ("H", "Qx", "Qy"):
        np.testing.assert_array_equal(st[k], ref[k], err_msg=k)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_members_equal_single_grid_runs(cuda, prec):
    cases = _cases()
    with Batch(prec, arena_bytes=ARENA) as b:
        slots = [b.add(c) for c in cases]
        b.run()
        for c, s in zip(cases, slots):
            t, dt, hmax, steps, state = b.status(s)
            n, t1, ref, mass = _alone(c, prec)
            assert state == FINISHED
            assert steps == n and t == t1, (c.name, steps, n, t, t1)
            _assert_same(b.state(s), ref)
            bt, bv, ba = b.mass_series(s)
            np.testing.assert_array_equal(bt, mass[0])
            np.testing.assert_allclose(bv, mass[1], rtol=1e-12, atol=1e-12)
            np.testing.assert_allclose(ba, mass[2], rtol=1e-12, atol=1e-9)


def test_fp64_batch_member_matches_oracle(cuda):
    case = _cases()[1]
    f = fc.pack(case)
    o = orc.OracleSim(case, f)
    n_ref = o.run(case.sim_time)
    ref = o.state()
    with Batch("f64", arena_bytes=ARENA) as b:
        s = b.add(case, f)
        b.add(_cases()[0])
        b.run()
        assert b.status(s)[3] == n_ref
        assert np.max(np.abs(b.state(s)["H"] - ref["H"])) <= 1e-9


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_strip_height_does_not_change_results(cuda, prec):
    case = _cases()[1]
    cls = size_class(case.nx, case.ny)
    out = []
    for rows, balance in ((1, 0), (3, 0), (8, 0), (64, 0), (64, 6)):
        with Batch(prec, arena_bytes=ARENA) as b:
            b.set_balance(balance)  # 0: fixed strip height; 6: re-cut as load changes
            b.set_rows(cls, rows)
            s = b.add(case)
            b.run()
            out.append(b.state(s))
    for st in out[1:]:
        _assert_same(st, out[0])


def test_result_alone_equals_result_in_a_changing_mix(cuda):
    """Continuous batching: the probe scenario joins while others are half
    way, others join and leave while it runs; its result is the one it has
    alone (bit for bit)."""
    cases = _cases()
    probe = cases[0]
    with Batch("f32", arena_bytes=ARENA) as b:
        s = b.add(probe)
        b.run()
        alone = b.state(s)
        n_alone = b.status(s)[3]
    with Batch("f32", arena_bytes=ARENA) as b:
        others = [b.add(c) for c in cases[1:3]]
        b.run(max_steps=40)
        s = b.add(probe)  # joins mid-run of the others
        b.launch(max_steps=25)
        late = b.add(cases[3])  # admitted while a launch is in flight
        b.sync()
        b.remove(others[0])  # leaves before finishing
        b.launch(max_steps=30)
        b.remove(others[1])  # removed while a launch is in flight
        b.sync()
        b.add(cases[4])
        b.run()
        assert b.status(s)[4] == FINISHED and b.status(late)[4] == FINISHED
        assert b.status(s)[3] == n_alone
        _assert_same(b.state(s), alone)


def test_admission_by_footprint(cuda):
    cases = _cases()
    with Batch("f32", arena_bytes=ARENA) as probe:
        need = [probe.footprint(c) for c in cases]
    order = np.argsort(need)
    a, c, bb = cases[order[-1]], cases[order[0]], cases[order[1]]  # largest, smallest, next
    na, nb, nc = need[order[-1]], need[order[1]], need[order[0]]
    arena = na + nb + nc // 2  # room for a and bb, not for c as well
    with Batch("f32", arena_bytes=arena) as b:
        s0 = b.try_add(a)
        s1 = b.try_add(bb)
        assert s0 is not None and s1 is not None
        assert b.try_add(c) is None  # refused, nothing changed
        assert b.info()["members"] == 2 and b.info()["arena_used"] == na + nb
        b.run()
        ref = b.state(s1)
        b.remove(s0)
        s2 = b.try_add(c)  # fits in the space a held
        assert s2 is not None
        b.run()
        assert b.status(s2)[4] == FINISHED
        _assert_same(b.state(s1), ref)  # a finished member is not stepped again
        n, _, st, _ = _alone(c, "f32")
        _assert_same(b.state(s2), st)


def test_stop_on_done_and_attention(cuda):
    cases = _cases()
    with Batch("f32", arena_bytes=ARENA) as b:
        short = b.add(cases[3], t_stop=60.0)
        long_ = b.add(cases[0])
        b.launch(stop_on_done=True)
        b.sync()
        assert b.status(short)[4] == FINISHED
        assert b.status(long_)[4] == RUNNING
        steps_before = b.info()["batch_steps"]
        b.launch()
        b.attention()
        b.sync()
        assert b.status(long_)[4] in (RUNNING, FINISHED)
        assert b.info()["batch_steps"] >= steps_before + 1
        b.run()
        assert b.status(long_)[4] == FINISHED
        n, t, st, _ = _alone(cases[0], "f32")
        _assert_same(b.state(long_), st)


def test_many_small_members(cuda):
    """More members than warps in one batch step's grid would hold at once
    (the active list spans several 32-wide compaction rounds)."""
    rng = np.random.default_rng(5)
    cases = [sc.small_case(int(rng.integers(12, 90)), int(rng.integers(12, 90)), seed=100 + k,
                           rain=bool(k % 2), sim_time=float(rng.uniform(60, 240)))
             for k in range(70)]
    with Batch("f32", arena_bytes=ARENA) as b:
        slots = [b.add(c) for c in cases]
        b.run()
        for k in (0, 33, 69):
            n, t, st, _ = _alone(cases[k], "f32")
            assert b.status(slots[k])[3] == n
            _assert_same(b.state(slots[k]), st)


def test_tuned_rows_are_candidates_and_leave_results_unchanged(cuda):
    """The autotuner returns one of its candidate heights per size class, with
    a measured rate for every candidate; a batch run with the tuned heights
    gives the same state as the scenario run alone."""
    from adaptflood_b200.tune import tune_rows
    scores = {}
    rows = tune_rows([12, 14], "f32", rows=(4, 8, 16), target_cells=1 << 20, steps=4,
                     warmup=1, arena_bytes=ARENA, scores_out=scores)
    assert set(rows) == {12, 14}
    for cls, r in rows.items():
        assert r in (4, 8, 16)
        assert set(scores[cls]) == {4, 8, 16}
        assert all(v > 0 for v in scores[cls].values())
    case = sc.small_case(90, 70, seed=41, rain=True, sim_time=200.0)
    n, t, st, _ = _alone(case, "f32")
    with Batch("f32", arena_bytes=ARENA, rows=rows) as b:
        s = b.add(case)
        b.run()
        assert b.status(s)[3] == n
        _assert_same(b.state(s), st)


def test_batch_step_limits_are_exact(cuda):
    """A batch launch takes exactly the batch steps asked for, whatever the
    number of steps per loop iteration."""
    cases = _cases()
    with Batch("f32", arena_bytes=ARENA) as b:
        slots = [b.add(c) for c in cases[:3]]
        total = 0
        for n in (1, 2, 3, 5, 6):
            b.launch(max_steps=n)
            b.sync()
            total += n
            assert b.info()["batch_steps"] == total
            assert all(b.status(s)[3] == total for s in slots)


def test_batch_trace_records_every_step(cuda):
    cases = _cases()[:3]
    with Batch("f32", arena_bytes=ARENA) as b:
        slots = [b.add(c) for c in cases]
        b.set_trace(100000)
        n = b.run()
        rec = b.trace()
        steps = [b.status(s)[3] for s in slots]
    assert rec.shape == (n, 4) and n == max(steps)
    start, end, cells, units = rec.T
    assert np.all(end >= start) and np.all(start[1:] >= end[:-1])
    # every member is active until it has taken its own steps
    want = [sum(c.cells for c, k in zip(cases, steps) if k > i) for i in range(n)]
    np.testing.assert_array_equal(cells, want)
    assert np.all(units > 0)
