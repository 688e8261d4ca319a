// af_common.cuh -- shared helpers for the AdaptFlood CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>
#include <mutex>

#include "adaptflood.h"

namespace af {

// Records the CUDA error text for af_last_cuda_error() and maps to AF_ECUDA.
int cuda_fail(cudaError_t e);

#define AF_CUDA(call)                              \
  do {                                             \
    cudaError_t af_e_ = (call);                    \
    if (af_e_ != cudaSuccess) return af::cuda_fail(af_e_); \
  } while (0)

#define AF_TRY(expr)              \
  do {                            \
    int af_rc_ = (expr);          \
    if (af_rc_ != AF_OK) return af_rc_; \
  } while (0)

constexpr int kSMs = 148;  // B200: 2 dies x 74 SMs

// Grid-stride launch size: a multiple of the SM count, capped by the work.
inline unsigned grid_for(long long n, int threads, int per_sm = 8) {
  long long need = (n + threads - 1) / threads;
  long long cap = (long long)kSMs * per_sm;
  if (need < 1) need = 1;
  return (unsigned)(need < cap ? need : cap);
}

// Monotone map of doubles onto unsigned 64-bit integers, so atomicMax on the
// image is a max on the doubles (negative values and -0.0 included).
__host__ __device__ inline unsigned long long ord_encode(double x) {
#ifdef __CUDA_ARCH__
  long long b = __double_as_longlong(x);
#else
  long long b;
  memcpy(&b, &x, 8);
#endif
  return b >= 0 ? ((unsigned long long)b | 0x8000000000000000ULL) : ~(unsigned long long)b;
}

__host__ __device__ inline double ord_decode(unsigned long long u) {
  unsigned long long b = (u & 0x8000000000000000ULL) ? (u & 0x7FFFFFFFFFFFFFFFULL) : ~u;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double x;
  memcpy(&x, &b, 8);
  return x;
#endif
}

// interpolate_bc_value / interpolate_rain (src/io.cpp:299-311, :88-100).  A
// linear scan that returns the first segment with times[i] <= t < times[i+1].
// When the series is non-decreasing (`sorted`), the same segment is the last
// index with times[i] <= t, found here by bisection.
__host__ __device__ inline double interp_series(const double* times, const double* vals, int n,
                                                double fixed, double t, bool sorted) {
  if (n == 0) return fixed;
  if (t <= times[0]) return vals[0];
  if (t >= times[n - 1]) return vals[n - 1];
  int i = -1;
  if (sorted) {
    if (!(t == t)) return vals[n - 1];  // NaN t: the linear scan matches no segment
    int lo = 0, hi = n - 1;  // invariant: times[lo] <= t < times[hi]
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (times[mid] <= t) lo = mid;
      else hi = mid;
    }
    i = lo;
  } else {
    for (int k = 0; k < n - 1; k++) {
      if (t >= times[k] && t < times[k + 1]) {
        i = k;
        break;
      }
    }
    if (i < 0) return vals[n - 1];
  }
  double ratio = (t - times[i]) / (times[i + 1] - times[i]);
  return vals[i] + ratio * (vals[i + 1] - vals[i]);
}

// Per-device scratch owned by the library: grows on demand, freed at exit.
struct Scratch {
  void* dev = nullptr;
  size_t bytes = 0;
  void* pinned = nullptr;  // 4 KB of pinned host memory for small readbacks
};
int scratch_get(size_t bytes, Scratch** out);  // current device; caller holds scratch_lock()
std::mutex& scratch_lock();

}  // namespace af
