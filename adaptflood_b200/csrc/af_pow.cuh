// af_pow.cuh -- the FP64 pow of the parity path, for host and device.
//
// The reference's friction term is pow(hflow, 10.0/3.0) (src/kernels.cpp:83,
// 133), evaluated by the C library of the machine it runs on.  CUDA's pow and
// glibc's (>= 2.28) differ in the last bit on a share of the depths, and
// those differences, divided by depths down to 1 mm in ComputeVelocity
// (src/kernels.cpp:293-351), reach 1e-9 m/s over a few hundred steps.  This
// is the published table-driven algorithm that glibc uses (Szabolcs Nagy's
// design for Arm Optimized Routines, adopted by glibc 2.28), restated:
//
//   log:  x = 2^k z, z in [0x1.69555p-1, 0x1.69555p0) split into 128
//         subintervals by the top bits of z; c is a point near the centre of
//         z's subinterval whose 1/c has few bits, so r = z/c - 1 = fma(z,1/c,-1)
//         is exact; log x = k ln2 + log c + log1p(r) as hi + lo, with
//         log1p(r) = r - r^2/2 + r^3 q(r) and the -r^2/2 term split exactly.
//   y*log x as ehi + elo (one fma for the product's error).
//   exp:  ehi = k ln2/128 + r, 2^(k/128) = 2^(k>>7) H_j (1 + T_j) from a
//         128-entry table, exp(r) = 1 + r + r^2 p(r); result
//         scale + scale*(T_j + r + r^2 p(r)), rounded once.
//
// The tables are generated from the algorithm's construction rule and the two
// polynomials are fitted by this project's own Remez exchange
// (gen_pow_tables.py -> af_pow_tables.h).  The multiply-adds that glibc's
// FMA build of this algorithm contracts are written as fma() here (AF_POW_FMA
// contraction points), every other operation rounds separately; translation
// units that include this file are compiled without FMA contraction.
//
// Domain: the fast path covers positive normal x with |y log x| in
// [2^-54, 512) -- every depth of a flood model; other arguments (zero,
// subnormal, negative, inf, nan, overflow and underflow) fall back to the
// platform's pow, whose special-value results are the same IEEE ones.
#pragma once

#include <stdint.h>
#include <string.h>

#include <cmath>

#include "af_pow_tables.h"

#ifdef __CUDACC__
#define AF_POW_HD __host__ __device__ __forceinline__
#else
#define AF_POW_HD inline
#endif

namespace af {
namespace pw {

struct LogEntry {
  double invc, logc, logctail, pad;
};
struct ExpEntry {
  uint64_t tail, sbits;
};

#define AF_POW_LOG_ENTRY(a, b, c) {a, b, c, 0.0},
#define AF_POW_EXP_ENTRY(a, b) {a, b},
// Host copies (the checker and host callers) and device copies (kernels).
static const LogEntry kLogHost[128] = {AF_POW_LOG_TABLE(AF_POW_LOG_ENTRY)};
static const ExpEntry kExpHost[128] = {AF_POW_EXP_TABLE(AF_POW_EXP_ENTRY)};
#ifdef __CUDACC__
static __device__ const LogEntry kLogDev[128] = {AF_POW_LOG_TABLE(AF_POW_LOG_ENTRY)};
static __device__ const ExpEntry kExpDev[128] = {AF_POW_EXP_TABLE(AF_POW_EXP_ENTRY)};
#endif
#undef AF_POW_LOG_ENTRY
#undef AF_POW_EXP_ENTRY

AF_POW_HD double as_double(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double d;
  memcpy(&d, &u, 8);
  return d;
#endif
}
AF_POW_HD uint64_t as_u64(double d) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u;
  memcpy(&u, &d, 8);
  return u;
#endif
}
AF_POW_HD double fma_d(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
// A multiply-add that glibc's FMA build contracts (AF_POW_CONTRACT 1) or
// rounds twice (0).
#ifndef AF_POW_CONTRACT
#define AF_POW_CONTRACT 1
#endif
AF_POW_HD double mad(double a, double b, double c) {
#if AF_POW_CONTRACT
  return fma_d(a, b, c);
#else
  return a * b + c;
#endif
}
AF_POW_HD LogEntry log_entry(int i) {
#ifdef __CUDA_ARCH__
  const double2 a = __ldg(reinterpret_cast<const double2*>(&kLogDev[i]));
  const double b = __ldg(&kLogDev[i].logctail);
  return LogEntry{a.x, a.y, b, 0.0};
#else
  return kLogHost[i];
#endif
}
AF_POW_HD ExpEntry exp_entry(int i) {
#ifdef __CUDA_ARCH__
  const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(&kExpDev[i]));
  return ExpEntry{v.x, v.y};
#else
  return kExpHost[i];
#endif
}

// log(x) = hi + lo for the 12-bit-exponent-adjusted bits ix of a positive
// normal x.
AF_POW_HD double log_hilo(uint64_t ix, double& lo_out) {
  const uint64_t tmp = ix - AF_POW_OFF;
  const int i = (int)((tmp >> 45) & 127);
  const int64_t k = (int64_t)tmp >> 52;  // arithmetic shift
  const uint64_t iz = ix - (tmp & (0xfffULL << 52));
  const double z = as_double(iz);
  const double kd = (double)k;
  const LogEntry e = log_entry(i);
  const double r = fma_d(z, e.invc, -1.0);  // exact: 1/c has few bits
  // k ln2 + log c + r (k*ln2hi + logc is exact)
  const double t1 = mad(kd, AF_POW_LN2HI, e.logc);
  const double t2 = t1 + r;
  const double lo1 = mad(kd, AF_POW_LN2LO, e.logctail);
  const double lo2 = t1 - t2 + r;
  // the -r^2/2 term, split into hi and its exact rounding error
  const double ar = AF_POW_A0 * r;
  const double ar2 = r * ar;
  const double ar3 = r * ar2;
  const double hi = t2 + ar2;
  const double lo3 = fma_d(ar, r, -ar2);
  const double lo4 = t2 - hi + ar2;
  // r^3 q(r), in the scaled form of the coefficients
  const double q = mad(ar2, mad(ar2, mad(r, AF_POW_A6, AF_POW_A5), mad(r, AF_POW_A4, AF_POW_A3)),
                       mad(r, AF_POW_A2, AF_POW_A1));
  const double lo = mad(ar3, q, lo1 + lo2 + lo3 + lo4);
  const double y = hi + lo;
  lo_out = hi - y + lo;
  return y;
}

// exp(x + xtail) for 2^-54 <= |x| < 512 (the caller checks the range).
AF_POW_HD double exp_hilo(double x, double xtail) {
  double kd = mad(AF_POW_INVLN2N, x, AF_POW_SHIFT);
  const uint64_t ki = as_u64(kd);
  kd -= AF_POW_SHIFT;
  double r = mad(kd, AF_POW_NEGLN2LON, mad(kd, AF_POW_NEGLN2HIN, x));
  r += xtail;
  const int idx = (int)(ki & 127);
  const uint64_t top = ki << 45;
  const ExpEntry e = exp_entry(idx);
  const double tail = as_double(e.tail);
  const uint64_t sbits = e.sbits + top;
  const double r2 = r * r;
  const double r4 = r2 * r2;
  const double tmp = mad(r4, mad(r, AF_POW_C5, AF_POW_C4),
                         mad(r2, mad(r, AF_POW_C3, AF_POW_C2), tail + r));
  const double scale = as_double(sbits);
  return mad(scale, tmp, scale);
}

// x^y for the parity path; see the header comment for the domain.
AF_POW_HD double pow_ref(double x, double y) {
  const uint64_t ix = as_u64(x);
  const uint32_t topx = (uint32_t)(ix >> 52);
  // positive normal x only (sign bit clear, exponent field 1..2046)
  if (topx - 1u < 0x7feu) {
    double lo;
    const double hi = log_hilo(ix, lo);
    const double ehi = y * hi;
    const double elo = mad(y, lo, fma_d(y, hi, -ehi));
    const uint32_t abstop = (uint32_t)(as_u64(ehi) >> 52) & 0x7ffu;
    // |ehi| in [2^-54, 512): the table path; below it exp(ehi) rounds to 1 + ehi
    if (abstop - 0x3c9u < 0x408u - 0x3c9u) return exp_hilo(ehi, elo);
    if (abstop < 0x3c9u) return 1.0 + ehi;
  }
#ifdef __CUDA_ARCH__
  return ::pow(x, y);
#else
  return std::pow(x, y);
#endif
}

}  // namespace pw
}  // namespace af
