"""The FP64 pow of the parity path (adaptflood_b200/csrc/af_pow.cuh).

The reference's friction term is the C library's pow(hflow, 10.0/3.0)
(src/kernels.cpp:83,133).  The library restates glibc's table-driven
algorithm; these tests pin the restatement to the C library of this machine
(glibc >= 2.28 with FMA: its pow is that algorithm) and the device build to
the host build.

Bars: on depths (1 mm .. 10 m, the flux law's range) and on a wide range, at
most 1e-6 of arguments may differ from the C library (measured about 1.3e-7,
each a single ulp); special values agree exactly; the device build equals the
host build bit for bit wherever the table path runs (|y log x| < 512: for
y = 10/3 every x between 1e-66 and 1e66).  Beyond that each build falls back
to its platform's pow (CUDA's on the device), which can differ from the C
library's in the last bit; no depth comes near that range.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "adaptflood_b200", "csrc")
Y = 10.0 / 3.0
MISMATCH_BAR = 1e-6


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _has_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return " fma " in f.read()
    except OSError:
        return False


def _samples(seed: int, n: int, lo: float, hi: float) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


SPECIAL = np.array([1.0, np.nextafter(1.0, 2.0), np.nextafter(1.0, 0.0), 0.0, -0.0, 5e-324,
                    2.2250738585072014e-308, 1e-310, np.inf, -np.inf, np.nan, -1.0, -0.5,
                    0.001, 10.0, 1e-100, 1e100, 1e300, 0.5, 2.0, 0.7057, 1.4114])


def _restated(x, y=Y):
    lib = orc.pow_check_lib()
    out = np.empty_like(x)
    lib.powc_restated(_p(x), _p(out), x.size, y)
    return out


def _libc(x, y=Y):
    lib = orc.pow_check_lib()
    out = np.empty_like(x)
    lib.powc_libc(_p(x), _p(out), x.size, y)
    return out


@pytest.mark.skipif(not _has_fma(), reason="the C library's pow takes its non-FMA variant here")
@pytest.mark.parametrize("seed,n,lo,hi", [(11, 20_000_000, 1e-3, 10.0),
                                          (12, 2_000_000, 1e-60, 1e60),
                                          (13, 2_000_000, 0.99, 1.01)])
def test_restated_pow_matches_the_c_library(seed, n, lo, hi):
    x = _samples(seed, n, lo, hi)
    bad = orc.pow_check_lib().powc_mismatch(_p(x), x.size, Y)
    assert bad <= MISMATCH_BAR * n, (bad, n)


def test_special_values_match_the_c_library():
    for y in (Y, 2.0, 0.5, -1.5):
        a, b = _libc(SPECIAL.copy(), y), _restated(SPECIAL.copy(), y)
        np.testing.assert_array_equal(a, b)


def test_tables_are_what_the_generator_writes():
    out = subprocess.run([sys.executable, os.path.join(CSRC, "gen_pow_tables.py")],
                         capture_output=True, text=True, check=True, cwd=CSRC).stdout
    with open(os.path.join(CSRC, "af_pow_tables.h")) as f:
        assert f.read() == out


@pytest.mark.gpu
def test_device_pow_equals_host_restatement(cuda):
    import torch
    from adaptflood_b200 import _lib
    x = np.concatenate([_samples(21, 1 << 22, 1e-3, 10.0), _samples(22, 1 << 18, 1e-60, 1e60),
                        SPECIAL])
    want = _restated(x)
    gx = torch.from_numpy(x).cuda()
    gout = torch.empty_like(gx)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().af_pow_eval(C.c_void_p(gx.data_ptr()), C.c_void_p(gout.data_ptr()), x.size,
                                Y, st)
    assert rc == _lib.AF_OK
    got = gout.cpu().numpy()
    np.testing.assert_array_equal(got, want)
    if _has_fma():
        libc = _libc(x)
        assert np.count_nonzero((got != libc) & ~(np.isnan(got) & np.isnan(libc))) <= \
            MISMATCH_BAR * x.size
