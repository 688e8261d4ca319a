// Kokkos_Core.hpp -- minimal host-only (OpenMP) stand-in for the subset of the
// Kokkos >= 4.0 API that AdaptFlood's src/kernels.cpp, src/io.cpp,
// src/async_output.cpp and src/main.cpp use.
//
// TEST INFRASTRUCTURE ONLY.  This header exists so the reference's own sources
// can be compiled unmodified on the CPU and act as the parity checker for the
// CUDA implementation.  Nothing in the shipped library includes it.
//
// API covered (grepped from the reference):
//   View<T*, Space>(label, n), operator()(i), data(), size(), extent(0)
//   create_mirror_view(v)       -- UVM views alias, so the mirror is the view
//   deep_copy(dst, src)         -- element copy (no-op when aliased)
//   parallel_for(label, n, f)   and  parallel_for(label, MDRangePolicy<Rank<2>>, f)
//   parallel_reduce(label, n, f, Max<double>(r))  and  (label, n, f, double& sum)
//   fence(), initialize(), finalize(), DefaultExecutionSpace, KOKKOS_LAMBDA,
//   KOKKOS_INLINE_FUNCTION, atomic_add, atomic_min.
//
// AF_SHIM_MANAGED: views in CudaUVMSpace are allocated with
// cudaMallocManaged, as Kokkos' CUDA backend does for that space, so the
// reference's main.cpp can be linked against a GPU implementation of
// src/kernels.hpp (the drop-in binding) while its inline loops keep touching
// the same arrays on the host.  Without it every view lives in host memory.
//
// Determinism notes:
//   * Max reductions are order independent, so FindHmax is exact.
//   * Sum reductions use a fixed static partition by thread id and combine the
//     per-thread partials in thread order: deterministic for a given
//     OMP_NUM_THREADS (the volume/area diagnostics only).
//   * 1-D ranges of at most kSerialBelow iterations run on one thread.  This
//     matters for main.cpp's point-source scatter, whose `H(idx) += ...` is not
//     atomic: with a serial loop two sources in one cell accumulate in file
//     order, which is the behaviour the CUDA implementation reproduces.
#ifndef AF_KOKKOS_SHIM_CORE_HPP
#define AF_KOKKOS_SHIM_CORE_HPP

#include <cfloat>
#include <cstddef>
#include <cstring>
#include <memory>
#include <string>
#include <typeinfo>
#include <vector>
#include <omp.h>
#ifdef AF_SHIM_MANAGED
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#endif

#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION

namespace Kokkos {

struct HostSpace {};
struct CudaUVMSpace {};
struct OpenMP {};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}
inline void fence() {}
inline void fence(const std::string&) {}

constexpr long kSerialBelow = 256;

template <class DataType, class Space = HostSpace>
class View;

// Storage of a view: host memory, or managed memory for CudaUVMSpace in the
// AF_SHIM_MANAGED build.  Zero-filled, as Kokkos value-initialises views.
template <class T, class Space>
struct ViewStore {
  std::vector<T> v;
  explicit ViewStore(size_t n) : v(n, T()) {}
  T* data() { return v.data(); }
};
#ifdef AF_SHIM_MANAGED
template <class T>
struct ViewStore<T, CudaUVMSpace> {
  T* p = nullptr;
  explicit ViewStore(size_t n) {
    if (cudaMallocManaged(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
      std::fprintf(stderr, "cudaMallocManaged of %zu bytes failed\n", n * sizeof(T));
      std::abort();
    }
    std::memset(p, 0, n * sizeof(T));
  }
  ~ViewStore() { cudaFree(p); }
  ViewStore(const ViewStore&) = delete;
  ViewStore& operator=(const ViewStore&) = delete;
  T* data() { return p; }
};
#endif

// Rank-1 view with shared (reference-counted) storage, so copies made by
// by-value lambda capture alias the same buffer, as Kokkos views do.
template <class T, class Space>
class View<T*, Space> {
 public:
  using value_type = T;
  using HostMirror = View<T*, Space>;

  View() = default;
  View(const std::string& label, size_t n)
      : label_(label), store_(std::make_shared<ViewStore<T, Space>>(n)), n_(n) {
    ptr_ = store_->data();
  }

  T& operator()(long i) const { return ptr_[i]; }
  T& operator[](long i) const { return ptr_[i]; }
  T* data() const { return ptr_; }
  size_t size() const { return n_; }
  size_t extent(int) const { return n_; }
  const std::string& label() const { return label_; }

 private:
  std::string label_;
  std::shared_ptr<ViewStore<T, Space>> store_;
  T* ptr_ = nullptr;
  size_t n_ = 0;
};

template <class V>
V create_mirror_view(const V& v) { return v; }

template <class V>
V create_mirror_view_and_copy(const HostSpace&, const V& v) { return v; }

template <class VD, class VS>
void deep_copy(const VD& dst, const VS& src) {
  if (dst.data() == src.data()) return;
  size_t n = dst.size() < src.size() ? dst.size() : src.size();
  std::memcpy(dst.data(), src.data(), n * sizeof(*dst.data()));
}

template <class T, class Space>
void deep_copy(const View<T*, Space>& dst, const T& value) {
  for (size_t i = 0; i < dst.size(); ++i) dst(i) = value;
}

template <unsigned N>
struct Rank {};

template <class R>
struct MDRangePolicy {
  long lo0, lo1, hi0, hi1;
  MDRangePolicy(std::initializer_list<long> lo, std::initializer_list<long> hi) {
    auto a = lo.begin();
    auto b = hi.begin();
    lo0 = a[0];
    lo1 = a[1];
    hi0 = b[0];
    hi1 = b[1];
  }
};

template <class F>
void parallel_for(const std::string&, long n, const F& f) {
  if (n <= 0) return;
  if (n <= kSerialBelow) {
    for (long i = 0; i < n; ++i) f((int)i);
    return;
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) f((int)i);
}

template <class F>
void parallel_for(long n, const F& f) { parallel_for(std::string(), n, f); }

template <class F, unsigned N>
void parallel_for(const std::string&, const MDRangePolicy<Rank<N>>& p, const F& f) {
  static_assert(N == 2, "only Rank<2> is used by the reference");
  if (p.hi0 <= p.lo0 || p.hi1 <= p.lo1) return;
  // Kokkos' default MDRange iteration is right-most index fastest; the
  // iterations are independent, so only the partition differs.
#pragma omp parallel for schedule(static)
  for (long j = p.lo1; j < p.hi1; ++j)
    for (long i = p.lo0; i < p.hi0; ++i) f((int)i, (int)j);
}

template <class T>
struct Max {
  T& ref;
  explicit Max(T& r) : ref(r) {}
  static T identity() { return -DBL_MAX; }
  static void join(T& dst, const T& src) {
    if (src > dst) dst = src;
  }
};

template <class F, class T>
void parallel_reduce(const std::string&, long n, const F& f, Max<T> red) {
  T result = Max<T>::identity();
  if (n > 0) {
    int nt = omp_get_max_threads();
    std::vector<T> part(nt, Max<T>::identity());
#pragma omp parallel num_threads(nt)
    {
      int tid = omp_get_thread_num();
      T local = Max<T>::identity();
#pragma omp for schedule(static)
      for (long i = 0; i < n; ++i) f((int)i, local);
      part[tid] = local;
    }
    for (int k = 0; k < nt; ++k) Max<T>::join(result, part[k]);
  }
  red.ref = result;
}

template <class F, class T>
void parallel_reduce(const std::string&, long n, const F& f, T& sum) {
  T result = T(0);
  if (n > 0) {
    int nt = omp_get_max_threads();
    std::vector<T> part(nt, T(0));
#pragma omp parallel num_threads(nt)
    {
      int tid = omp_get_thread_num();
      T local = T(0);
#pragma omp for schedule(static)
      for (long i = 0; i < n; ++i) f((int)i, local);
      part[tid] = local;
    }
    for (int k = 0; k < nt; ++k) result += part[k];
  }
  sum = result;
}

template <class T>
inline void atomic_add(T* p, T v) {
#pragma omp atomic
  *p += v;
}

template <class T>
inline void atomic_min(T* p, T v) {
#pragma omp critical(af_kokkos_shim_atomic_min)
  {
    if (v < *p) *p = v;
  }
}

}  // namespace Kokkos

#endif  // AF_KOKKOS_SHIM_CORE_HPP
