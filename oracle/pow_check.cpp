// pow_check.cpp -- CPU checker of the FP64 pow on the parity path (test
// infrastructure only).
//
// The reference evaluates pow(hflow, 10.0/3.0) with the C library
// (src/kernels.cpp:83,133).  This library exposes, over arrays, (1) that
// C-library pow and (2) the host build of the library's restatement in
// adaptflood_b200/csrc/af_pow.cuh, so tests can compare the two with each
// other and with the device build (af_pow_eval).  Built with FMA instructions
// available (the restatement's fused multiply-adds are exact either way) and
// without contraction of any other expression.
#include <cmath>

#include "af_pow.cuh"

extern "C" {

void powc_libc(const double* x, double* out, long n, double y) {
  volatile double yy = y;  // a run-time exponent: the call is never folded
  for (long i = 0; i < n; i++) out[i] = pow(x[i], yy);
}

void powc_restated(const double* x, double* out, long n, double y) {
  for (long i = 0; i < n; i++) out[i] = af::pw::pow_ref(x[i], y);
}

long powc_mismatch(const double* x, long n, double y) {
  volatile double yy = y;
  long bad = 0;
  for (long i = 0; i < n; i++) {
    const double a = pow(x[i], yy);
    const double b = af::pw::pow_ref(x[i], y);
    if (!(a == b || (a != a && b != b))) bad++;
  }
  return bad;
}
}
