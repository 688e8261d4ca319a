"""Compile the CUDA library in-tree: adaptflood_b200/libadaptflood.so (sm_100a).

Floating-point flags per translation unit:
  * af_plain.cu, af_step_f64.cu, af_sim.cu: -fmad=false, so FP64 expressions
    round exactly as the reference's C++ does on the CPU;
  * af_step_f32.cu: -use_fast_math (FP32 path: FMA contraction, approximate
    division/sqrt and SFU exp2/log2 are within its error budget).  The flag
    also lets the compiler contract the FP64 bookkeeping compiled in this unit
    for the FP32 kernels (time t + dt, the CFL dt, hydrograph and rain
    interpolation, the compensated volume sums) into fused multiply-adds: those
    FP64 values may differ from the FP64 path's in the last bit, far inside the
    FP32 path's tolerance, and the same in its single-grid and batch kernels.
Host code is compiled with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libadaptflood.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++"
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-ffp-contract=off", "-ccbin", HOSTCXX, "-I", INCLUDE, "-I", CSRC]
EXACT = ["-fmad=false"]
FAST = ["-use_fast_math"]

UNITS = [
    ("af_plain.cu", EXACT),
    ("af_step_f64.cu", EXACT),
    ("af_step_f32.cu", FAST),
    ("af_sim.cu", EXACT),
    ("af_batch.cu", EXACT),
    ("af_xfer.cu", EXACT),
]
HOST_UNITS = ["af_io.cpp", "af_arena.cpp", "af_output.cpp"]
HEADERS = ["af_common.cuh", "af_pow.cuh", "af_pow_tables.h", "af_step.cuh", "af_simcore.cuh", "af_arena.h", "af_output.h",
           "af_xfer.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, ptxas_info: bool = False, obj_dir: str = None, lib: str = None,
          defines=()) -> str:
    """Compiles the library; obj_dir/lib/defines build an alternative
    configuration elsewhere (the default is the in-tree library)."""
    OBJ = obj_dir or globals()["OBJ"]
    LIB = lib or globals()["LIB"]
    dflags = [f"-D{d}" for d in defines]
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "adaptflood.h")]
    jobs = []
    objs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if ptxas_info or _newer(o, [s, __file__] + hdrs):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC, *ARCH, *COMMON, *flags, *dflags, *extra, "-c", s, "-o", o])
    for src in HOST_UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _newer(o, [s, __file__] + hdrs):
            jobs.append([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread",
                         "-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o])
    log = []
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for out in ex.map(_run, jobs):
            log.append(out)
    if jobs or not os.path.exists(LIB):
        log.append(_run([NVCC, *ARCH, "-shared", "-ccbin", HOSTCXX, "-o", LIB, *objs,
                         "-lcudart", "-lcudadevrt"]))
    text = "".join(log)
    if verbose:
        print(text)
    return text


# A test build whose ring waits give up at once (AF_RING_WAIT_LIMIT=0): the
# failure tests run the kernels' time-out path with it (the warp drains its
# copies, flags the control block, and the loop stops with AF_ESTATE).
WAITTEST_LIB = os.path.join(HERE, "libadaptflood_waittest.so")


def build_wait_test(verbose: bool = False) -> str:
    return build(verbose=verbose, obj_dir=os.path.join(HERE, "_build_waittest"), lib=WAITTEST_LIB,
                 defines=("AF_RING_WAIT_LIMIT=0",))


if __name__ == "__main__":
    print(build(verbose=False, ptxas_info="--ptxas" in sys.argv) or "up to date")
