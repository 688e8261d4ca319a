"""af_add_point_sources_noalloc: the point-source scatter for callers that
cannot let the library allocate device memory (they own all of it through
their own pool, or cannot afford the device-wide synchronisation of cudaFree).

Checked through the C ABI against af_add_point_sources on the same inputs,
bit for bit, on two calls in a row (the calls share one fixed device array,
so the second call must not see anything the first left behind), and against
the reference's sequential scatter (src/main.cpp:256-260 in file order)
computed on the CPU.  This file is collected last on purpose; it passes
alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from adaptflood_b200 import _lib

pytestmark = pytest.mark.gpu


def _call(fn, H, idx, flow, n, ncells):
    import torch
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return fn(C.c_void_p(H.data_ptr()), C.c_void_p(idx.data_ptr()), C.c_void_p(flow.data_ptr()),
              n, ncells, st)


def _case(seed, n, ncell, bad=False):
    import torch
    rng = np.random.default_rng(seed)
    H = rng.uniform(0.0, 0.3, ncell)
    idx = rng.integers(0, max(2, ncell // 4), n).astype(np.int32)  # many shared cells
    if bad:
        idx[n // 3] = ncell + 7
    flow = rng.normal(0.0, 0.08, n)
    return (torch.from_numpy(H).cuda(), torch.from_numpy(idx).cuda(),
            torch.from_numpy(flow).cuda())


def _sequential(H, idx, flow, ncell):
    """The reference's scatter, one source after another in file order,
    skipping indices off the grid."""
    out = H.copy()
    for k in range(idx.size):
        i = int(idx[k])
        if 0 <= i < ncell:
            out[i] += flow[k]
            if out[i] < 0.0:
                out[i] = 0.0
    return out


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(cuda):
    lib = _lib.lib()
    max_n = 4096
    for seed, n, ncell, bad in ((1, max_n, 5003, False), (2, 37, 211, True), (3, 1, 9, False),
                                (4, 1999, 777, False)):
        H0, idx, flow = _case(seed, n, ncell, bad)
        want = H0.clone()
        rc_want = _call(lib.af_add_point_sources, want, idx, flow, n, ncell)
        got = H0.clone()
        rc_got = _call(lib.af_add_point_sources_noalloc, got, idx, flow, n, ncell)
        assert rc_got == rc_want == (_lib.AF_ERANGE if bad else _lib.AF_OK)
        assert bool((got == want).all()), f"seed {seed}"
        seq = _sequential(H0.cpu().numpy(), idx.cpu().numpy(), flow.cpu().numpy(), ncell)
        np.testing.assert_array_equal(got.cpu().numpy(), seq)


def test_noalloc_rejects_more_than_the_maximum(cuda):
    lib = _lib.lib()
    H0, idx, flow = _case(5, 4097, 300)
    H = H0.clone()
    assert _call(lib.af_add_point_sources_noalloc, H, idx, flow, 4097, 300) == _lib.AF_ERANGE
    assert bool((H == H0).all())
    # the array is still usable afterwards
    H1, idx1, flow1 = _case(6, 64, 50)
    a, b = H1.clone(), H1.clone()
    assert _call(lib.af_add_point_sources, a, idx1, flow1, 64, 50) == _lib.AF_OK
    assert _call(lib.af_add_point_sources_noalloc, b, idx1, flow1, 64, 50) == _lib.AF_OK
    assert bool((a == b).all())
