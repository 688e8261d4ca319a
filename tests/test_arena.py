"""The batch's arena planner (host logic, no device): placements never
overlap, stay aligned and inside the arena, a refused request changes
nothing, releases coalesce, and best fit picks the smallest hole."""
import numpy as np
import pytest

from adaptflood_b200 import _lib
from adaptflood_b200.batch import Arena

ALIGN = 256


def _up(n):
    return (max(n, 1) + ALIGN - 1) // ALIGN * ALIGN


def test_random_alloc_free_matches_a_model():
    rng = np.random.default_rng(7)
    size = 1 << 24
    a = Arena(size)
    live = {}  # off -> len
    for it in range(4000):
        if live and rng.random() < 0.45:
            off = int(rng.choice(list(live)))
            a.free(off)
            del live[off]
        else:
            n = int(rng.integers(1, 1 << 19))
            off = a.alloc(n)
            used_before = sum(live.values())
            if off is None:
                # refused: no hole of _up(n) exists in the model either
                ivs = sorted(live.items())
                holes, at = [], 0
                for o, ln in ivs:
                    holes.append(o - at)
                    at = o + ln
                holes.append(size - at)
                assert max(holes) < _up(n)
                assert a.stats()[0] == used_before
                continue
            assert off % ALIGN == 0 and off + _up(n) <= size
            for o, ln in live.items():
                assert off + _up(n) <= o or o + ln <= off, "overlap"
            live[off] = _up(n)
        used, largest, blocks = a.stats()
        assert used == sum(live.values())
        assert blocks == len(live)
    for off in list(live):
        a.free(off)
    assert a.stats() == (0, size, 0)  # everything coalesced back into one block


def test_best_fit_and_coalescing():
    a = Arena(10 * ALIGN)
    offs = [a.alloc(ALIGN) for _ in range(10)]
    assert offs == [k * ALIGN for k in range(10)]
    assert a.alloc(1) is None
    a.free(offs[1])                     # hole of 1
    a.free(offs[4]); a.free(offs[5]); a.free(offs[6])  # hole of 3
    assert a.stats()[1] == 3 * ALIGN
    assert a.alloc(ALIGN) == offs[1]    # the 1-block hole, not the 3-block one
    assert a.alloc(2 * ALIGN) == offs[4]
    assert a.alloc(2 * ALIGN) is None   # only one block left
    a.free(offs[4])                     # merges with the free block after it
    assert a.stats()[1] == 3 * ALIGN
    with pytest.raises(_lib.AFError):
        a.free(6 * ALIGN)               # free space, not an allocated block
    with pytest.raises(_lib.AFError):
        a.free(12345)


def test_invalid_arguments():
    lib = _lib.lib()
    assert lib.af_arena_create(16, None) == _lib.AF_EINVAL
    assert lib.af_arena_alloc(None, 16, None) == _lib.AF_EINVAL
    a = Arena(0)
    assert a.alloc(1) is None
