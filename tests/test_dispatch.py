"""Multi-GPU ensembles by host dispatch (adaptflood_b200.dispatch): balanced
shares, and two gloo ranks on the CPU that run their shares with a host-only
stand-in batch and gather every scenario's outcome exactly once."""
import math
import os
import pickle
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from adaptflood_b200 import dispatch
from adaptflood_b200 import scenarios as sc


def _cases(n=23, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx, ny = int(rng.integers(8, 90)), int(rng.integers(8, 90))
        out.append(sc.Case(nx, ny, float(rng.choice([2.0, 5.0, 10.0])), np.zeros((ny, nx)),
                           sim_time=float(rng.uniform(50, 900)), name=f"s{k}"))
    return out


def test_partition_is_balanced_and_complete():
    rng = np.random.default_rng(1)
    work = list(rng.lognormal(0, 1.0, 200))
    for world in (1, 2, 3, 8):
        shares = dispatch.partition(work, world)
        assert sorted(k for s in shares for k in s) == list(range(len(work)))
        loads = [sum(work[k] for k in s) for s in shares]
        lower = max(sum(work) / world, max(work))  # no split can beat this
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9
    with pytest.raises(ValueError):
        dispatch.partition(work, 0)


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _fakes import FakeBatch
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        res = dispatch.run_ensemble(_cases(), rank, world, dist,
                                    batch_factory=lambda: FakeBatch(arena_bytes=1 << 30, dt=7.0))
        with open(os.path.join(out_dir, f"r{rank}.pkl"), "wb") as f:
            pickle.dump(res, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_run_their_shares_and_gather_all(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    cases = _cases()
    shares = dispatch.partition([dispatch.work_estimate(c) for c in cases], world)
    for r in range(world):
        res = pickle.load(open(tmp_path / f"r{r}.pkl", "rb"))
        assert sorted(res) == list(range(len(cases)))  # every scenario, once, on every rank
        for k, v in res.items():
            assert v["rank"] == next(q for q in range(world) if k in shares[q])
            assert v["steps"] == math.ceil(cases[k].sim_time / 7.0) and v["state"] == 1


class _FailingBatch:
    """A batch whose admission fails (as Batch.add does when the device
    refuses), on one rank only."""

    def try_add(self, case, forcing=None, t_stop=None):
        raise RuntimeError("admission failed on purpose")

    def close(self):
        pass


def _rank_fail_main(rank, world, port, out_dir):
    import sys
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _fakes import FakeBatch
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        factory = (lambda: _FailingBatch()) if rank == 1 else (
            lambda: FakeBatch(arena_bytes=1 << 30, dt=7.0))
        try:
            dispatch.run_ensemble(_cases(), rank, world, dist, batch_factory=factory)
            msg = "returned"
        except RuntimeError as e:
            msg = str(e)
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(msg)
    finally:
        dist.destroy_process_group()


def test_a_failing_rank_makes_every_rank_raise(tmp_path):
    import time
    world = 2
    t0 = time.time()
    mp.spawn(_rank_fail_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    assert time.time() - t0 < 50  # well inside the process group's timeout
    for r in range(world):
        msg = open(tmp_path / f"r{r}.txt").read()
        assert "rank 1: RuntimeError: admission failed on purpose" in msg


def test_a_share_larger_than_the_arena_runs_in_waves():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _fakes import FakeBatch
    cases = _cases()
    biggest = max(c.cells for c in cases) * 28
    fb = FakeBatch(arena_bytes=3 * biggest, dt=7.0)
    res = dispatch.run_ensemble(cases, 0, 1, None, batch_factory=lambda: fb)
    assert sorted(res) == list(range(len(cases)))
    for k, v in res.items():
        assert v["steps"] == math.ceil(cases[k].sim_time / 7.0) and v["state"] == 1
    assert fb.peak_used <= 3 * biggest and not fb.slots  # every slot freed
    with pytest.raises(MemoryError):
        dispatch.run_ensemble(cases, 0, 1, None,
                              batch_factory=lambda: FakeBatch(arena_bytes=biggest // 2, dt=7.0))
