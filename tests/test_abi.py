"""The C ABI library loads and exports every entry point include/*.h declares;
argument validation that needs no device."""
import ctypes as C
import glob
import os
import re

from adaptflood_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        names |= set(re.findall(r"\b(af_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 28
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert declared_symbols() <= set(_lib._SIGS)


def test_strerror_and_version():
    lib = _lib.lib()
    assert lib.af_strerror(0) == b"ok"
    assert lib.af_strerror(-2) == b"index or size out of range"
    assert lib.af_version() >= 10000


def test_validation_without_device():
    lib = _lib.lib()
    assert lib.af_update_qs(None, None, None, None, -1, 4, 1.0, None) == _lib.AF_EINVAL
    assert lib.af_update_qs(None, None, None, None, 65535, 65535, 1.0, None) == _lib.AF_ERANGE
    assert lib.af_fill(None, -5, 0.0, None) == _lib.AF_EINVAL
    assert lib.af_fill(None, 0, 0.0, None) == _lib.AF_OK
    assert lib.af_pow_eval(None, None, -1, 2.0, None) == _lib.AF_EINVAL
    assert lib.af_pow_eval(None, None, 0, 2.0, None) == _lib.AF_OK
    assert lib.af_add_point_sources(None, None, None, 0, 10, None) == _lib.AF_OK
    assert lib.af_apply_point_bcs(None, None, None, None, -1, 0, 1.0, 1.0, 1.0, 10,
                                  None) == _lib.AF_EINVAL
    assert lib.af_sim_create(None, None, None, None, 0, 0, None) == _lib.AF_EINVAL
    d = _lib.CaseDesc()
    d.nx, d.ny, d.dx, d.theta = 1, 5, 1.0, 1.0  # one column: rejected
    f = _lib.ForcingDesc()
    dem = (C.c_double * 5)()
    h = C.c_void_p()
    assert lib.af_sim_create(C.byref(d), C.byref(f), dem, None, 0, 0, C.byref(h)) == _lib.AF_EINVAL
    d.nx, d.theta = 5, 0.5  # theta != 1: the fused step implements the reference's theta = 1
    assert lib.af_sim_create(C.byref(d), C.byref(f), dem, None, 0, 0, C.byref(h)) == _lib.AF_EINVAL
