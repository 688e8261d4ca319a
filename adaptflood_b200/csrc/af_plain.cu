// af_plain.cu -- the drop-in layer: one CUDA kernel per function of the
// reference's src/kernels.hpp, FP64, reference layout, synchronous calls.
//
// Compiled with -fmad=false: every expression below rounds exactly as the
// reference's C++ does on the CPU.  The friction term's pow(hflow, 10/3)
// (src/kernels.cpp:83,133) is the C library's table-driven algorithm restated
// in af_pow.cuh, which returns glibc's value on all but ~1e-7 of arguments.
#include <cub/device/device_radix_sort.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "af_common.cuh"
#include "af_pow.cuh"

namespace af {

namespace {
thread_local char g_last_cuda_error[256] = "";

struct DevScratch {
  Scratch s[64];
};
DevScratch g_scratch;
std::mutex g_scratch_mu;

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool face_count_ok(int xsz, int ysz) {
  return (long long)(xsz + 1) * (long long)(ysz + 1) <= 0x7FFFFFFFLL;
}
}  // namespace

int cuda_fail(cudaError_t e) {
  snprintf(g_last_cuda_error, sizeof(g_last_cuda_error), "%s: %s", cudaGetErrorName(e),
           cudaGetErrorString(e));
  return AF_ECUDA;
}

std::mutex& scratch_lock() { return g_scratch_mu; }

int scratch_get(size_t bytes, Scratch** out) {
  int dev = 0;
  AF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return AF_EINVAL;
  Scratch& s = g_scratch.s[dev];
  if (!s.pinned) AF_CUDA(cudaMallocHost(&s.pinned, 4096));
  if (s.bytes < bytes) {
    if (s.dev) AF_CUDA(cudaFree(s.dev));
    s.dev = nullptr;
    s.bytes = 0;
    size_t want = bytes < (1u << 20) ? (1u << 20) : bytes;
    cudaError_t e = cudaMalloc(&s.dev, want);
    if (e != cudaSuccess) {
      cuda_fail(e);
      return AF_ENOMEM;
    }
    s.bytes = want;
  }
  *out = &s;
  return AF_OK;
}

// ------------------------------------------------------------ reductions
__device__ inline double warp_max(double m) {
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_down_sync(0xffffffffu, m, o);
    if (v > m) m = v;
  }
  return m;
}

// FindHmax of src/kernels.cpp:30-33: max H over cells with DEM != nodata.
__global__ void k_hmax(const double* __restrict__ H, const double* __restrict__ DEM, long long n,
                       double nodata, unsigned long long* __restrict__ acc) {
  double m = -DBL_MAX;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double h = H[i];
    if (DEM[i] != nodata && h > m) m = h;
  }
  m = warp_max(m);
  __shared__ double sm[32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sm[w] = m;
  __syncthreads();
  if (w == 0) {
    m = lane < (int)(blockDim.x >> 5) ? sm[lane] : -DBL_MAX;
    m = warp_max(m);
    if (lane == 0) atomicMax(acc, ord_encode(m));
  }
}

__global__ void k_set_u64(unsigned long long* p, unsigned long long v) { *p = v; }

// ------------------------------------------------------------ face fluxes
// getmax / getmin of src/types.hpp:14-15 (not fmax/fmin: NaN and signed-zero
// operands must pick the same side as the reference).
__device__ inline double gmax(double a, double b) { return (a > b) ? a : b; }
__device__ inline double gmin(double a, double b) { return (a < b) ? a : b; }

// Qx of src/kernels.cpp:46-93, one thread per interior x-face.
__global__ void k_qx(const double* __restrict__ H, const double* __restrict__ DEM,
                     double* __restrict__ Qx, const double* __restrict__ Qxold,
                     const double* __restrict__ Qyold, int xsz, int ysz, double dx, double FPn,
                     double DepthThresh, double MaxHflow, double dt, double g, double theta,
                     double nodata) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= xsz - 1 || j >= ysz) return;
  int p0 = i + j * xsz, p1 = i + 1 + j * xsz;
  int pq0 = (i + 1) + j * (xsz + 1);
  double z0 = DEM[p0], z1 = DEM[p1];
  if (z0 == nodata || z1 == nodata) {
    Qx[pq0] = 0.0;
    return;
  }
  double h0 = H[p0], h1 = H[p1];
  double fn = FPn;
  double y0 = z0 + h0, y1 = z1 + h1;
  double dh = y0 - y1;
  double Sf = -dh / dx;
  double hflow = gmax(y0, y1) - gmax(z0, z1);
  hflow = gmax(hflow, 0.0);
  hflow = gmin(hflow, MaxHflow);
  double Q = 0.0;
  if (hflow > DepthThresh) {
    double q0 = Qxold[pq0];
    double qup = (i > 0) ? Qxold[pq0 - 1] : 0.0;
    double qdown = (i < xsz - 2) ? Qxold[pq0 + 1] : 0.0;
    int pqy1 = i + j * (xsz + 1);
    int pqy2 = (i + 1) + j * (xsz + 1);
    int pqy3 = i + (j + 1) * (xsz + 1);
    int pqy4 = (i + 1) + (j + 1) * (xsz + 1);
    double qy_avg = (Qyold[pqy1] + Qyold[pqy2] + Qyold[pqy3] + Qyold[pqy4]) / 4.0;
    double qvect = sqrt(q0 * q0 + qy_avg * qy_avg);
    double numerator = (theta * q0 + 0.5 * (1.0 - theta) * (qup + qdown)) - (g * dt * hflow * Sf);
    double denominator = 1.0 + g * dt * hflow * fn * fn * fabs(qvect) / pw::pow_ref(hflow, 10.0 / 3.0);
    Q = numerator / denominator * dx;
    if (Q * dh < 0.0) {
      numerator = q0 - (g * dt * hflow * Sf);
      Q = numerator / denominator * dx;
    }
  }
  Qx[pq0] = Q;
}

// Qy of src/kernels.cpp:96-143, one thread per interior y-face.
__global__ void k_qy(const double* __restrict__ H, const double* __restrict__ DEM,
                     double* __restrict__ Qy, const double* __restrict__ Qxold,
                     const double* __restrict__ Qyold, int xsz, int ysz, double dx, double FPn,
                     double DepthThresh, double MaxHflow, double dt, double g, double theta,
                     double nodata) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= xsz || j >= ysz - 1) return;
  int p0 = i + j * xsz, p1 = i + (j + 1) * xsz;
  int pq0 = i + (j + 1) * (xsz + 1);
  double z0 = DEM[p0], z1 = DEM[p1];
  if (z0 == nodata || z1 == nodata) {
    Qy[pq0] = 0.0;
    return;
  }
  double h0 = H[p0], h1 = H[p1];
  double fn = FPn;
  double y0 = z0 + h0, y1 = z1 + h1;
  double dh = y0 - y1;
  double Sf = -dh / dx;
  double hflow = gmax(y0, y1) - gmax(z0, z1);
  hflow = gmax(hflow, 0.0);
  hflow = gmin(hflow, MaxHflow);
  double Q = 0.0;
  if (hflow > DepthThresh) {
    double q0 = Qyold[pq0];
    double qup = (j > 0) ? Qyold[i + j * (xsz + 1)] : 0.0;
    double qdown = (j < ysz - 2) ? Qyold[i + (j + 2) * (xsz + 1)] : 0.0;
    int pqx1 = i + j * (xsz + 1);
    int pqx2 = (i + 1) + j * (xsz + 1);
    int pqx3 = i + (j + 1) * (xsz + 1);
    int pqx4 = (i + 1) + (j + 1) * (xsz + 1);
    double qx_avg = (Qxold[pqx1] + Qxold[pqx2] + Qxold[pqx3] + Qxold[pqx4]) / 4.0;
    double qvect = sqrt(q0 * q0 + qx_avg * qx_avg);
    double numerator = (theta * q0 + 0.5 * (1.0 - theta) * (qup + qdown)) - (g * dt * hflow * Sf);
    double denominator = 1.0 + g * dt * hflow * fn * fn * fabs(qvect) / pw::pow_ref(hflow, 10.0 / 3.0);
    Q = numerator / denominator * dx;
    if (Q * dh < 0.0) {
      numerator = q0 - (g * dt * hflow * Sf);
      Q = numerator / denominator * dx;
    }
  }
  Qy[pq0] = Q;
}

// BCs_GPU of src/kernels.cpp:149-256; blockIdx.y selects the side (W, E, N, S).
__global__ void k_bcs(double* __restrict__ Qx, double* __restrict__ Qy,
                      const double* __restrict__ H, const double* __restrict__ DEM, int xsz,
                      int ysz, double dx, double g, double nodata, int wf, int ef, int nf,
                      int sf) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int side = blockIdx.y;
  if (side == 0) {  // west, face (0, j)
    if (wf) {
      if (k >= ysz) return;
      int j = k;
      int p0 = 0 + j * xsz;
      double h0 = H[p0], z0 = DEM[p0];
      double Q = 0.0;
      if (!(z0 == nodata || h0 < 0.001)) {
        int p1 = 1 + j * xsz;
        double h1 = H[p1], z1 = DEM[p1];
        double y0 = z0 + h0, y1 = z1 + h1;
        if (y0 > z0) {
          double Sf = (y1 - y0) / dx;
          if (Sf < 0) Q = -h0 * sqrt(g * h0) * dx * 0.5;
        }
      }
      Qx[j * (xsz + 1)] = Q;
    } else {
      if (k >= ysz + 1) return;
      Qx[k * (xsz + 1)] = 0.0;
    }
  } else if (side == 1) {  // east, face (xsz, j)
    if (ef) {
      if (k >= ysz) return;
      int j = k;
      int p0 = (xsz - 1) + j * xsz;
      double h0 = H[p0], z0 = DEM[p0];
      double Q = 0.0;
      if (!(z0 == nodata || h0 < 0.001) && h0 > 0.001) Q = h0 * sqrt(g * h0) * dx * 0.5;
      Qx[xsz + j * (xsz + 1)] = Q;
    } else {
      if (k >= ysz + 1) return;
      Qx[xsz + k * (xsz + 1)] = 0.0;
    }
  } else if (side == 2) {  // north, face (i, 0)
    if (nf) {
      if (k >= xsz) return;
      double h0 = H[k], z0 = DEM[k];
      double Q = 0.0;
      if (!(z0 == nodata || h0 < 0.001) && h0 > 0.001) Q = -h0 * sqrt(g * h0) * dx * 0.5;
      Qy[k] = Q;
    } else {
      if (k >= xsz + 1) return;
      Qy[k] = 0.0;
    }
  } else {  // south, face (i, ysz)
    if (sf) {
      if (k >= xsz) return;
      int p0 = k + (ysz - 1) * xsz;
      double h0 = H[p0], z0 = DEM[p0];
      double Q = 0.0;
      if (!(z0 == nodata || h0 < 0.001) && h0 > 0.001) Q = h0 * sqrt(g * h0) * dx * 0.5;
      Qy[k + ysz * (xsz + 1)] = Q;
    } else {
      if (k >= xsz + 1) return;
      Qy[k + ysz * (xsz + 1)] = 0.0;
    }
  }
}

// UpdateH of src/kernels.cpp:280-290.
__global__ void k_update_h(double* __restrict__ H, const double* __restrict__ Qx,
                           const double* __restrict__ Qy, int xsz, int ysz, double dA,
                           double Tstep) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= xsz || j >= ysz) return;
  int idx = i + j * xsz;
  double Qx_in = Qx[i + j * (xsz + 1)], Qx_out = Qx[(i + 1) + j * (xsz + 1)];
  double Qy_in = Qy[i + j * (xsz + 1)], Qy_out = Qy[i + (j + 1) * (xsz + 1)];
  double h = H[idx] + Tstep * (Qx_in - Qx_out + Qy_in - Qy_out) / dA;
  if (h < 0.0) h = 0.0;
  H[idx] = h;
}

// ComputeVx / ComputeVy of src/kernels.cpp:296-348.
__global__ void k_velocity(double* __restrict__ Vx, double* __restrict__ Vy,
                           const double* __restrict__ H, const double* __restrict__ DEM,
                           const double* __restrict__ Qx, const double* __restrict__ Qy, int xsz,
                           int ysz, double dx, double nodata) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= xsz || j >= ysz) return;
  int idx = i + j * xsz;
  double z = DEM[idx], h = H[idx];
  if (z == nodata || h < 0.001) {
    Vx[idx] = 0.0;
    Vy[idx] = 0.0;
    return;
  }
  double hflow = h;
  if (hflow < 0.001) hflow = 0.001;
  double ql = Qx[i + j * (xsz + 1)], qr = Qx[(i + 1) + j * (xsz + 1)];
  double vl = (fabs(ql) > 1e-10) ? ql / dx / hflow : 0.0;
  double vr = (fabs(qr) > 1e-10) ? qr / dx / hflow : 0.0;
  Vx[idx] = (fabs(vl) > fabs(vr)) ? vl : vr;
  double qt = Qy[i + j * (xsz + 1)], qb = Qy[i + (j + 1) * (xsz + 1)];
  double vt = (fabs(qt) > 1e-10) ? qt / dx / hflow : 0.0;
  double vb = (fabs(qb) > 1e-10) ? qb / dx / hflow : 0.0;
  Vy[idx] = (fabs(vt) > fabs(vb)) ? vt : vb;
}

// Rainfall of src/kernels.cpp:360-365.
__global__ void k_rain(double* __restrict__ H, const double* __restrict__ DEM, long long n,
                       double rain_depth, double nodata) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (DEM[i] != nodata) {
      double h = H[i] + rain_depth;
      if (h < 0.0) h = 0.0;
      H[i] = h;
    }
  }
}

// UpdateQxold / UpdateQyold of src/kernels.cpp:10-16.
__global__ void k_update_qs(const double* __restrict__ Qx, const double* __restrict__ Qy,
                            double* __restrict__ Qxold, double* __restrict__ Qyold, long long f,
                            double dxinv) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < f;
       k += (long long)gridDim.x * blockDim.x) {
    Qxold[k] = Qx[k] * dxinv;
    Qyold[k] = Qy[k] * dxinv;
  }
}

__global__ void k_fill(double* __restrict__ x, long long n, double v) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    x[k] = v;
}

// The parity path's pow (af_pow.cuh) over an array, for checking it against
// the C library's on the host.
__global__ void k_pow_eval(const double* __restrict__ x, double* __restrict__ out, int64_t n,
                           double y) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    out[k] = pw::pow_ref(x[k], y);
}

// Vol / Area of src/main.cpp:293-298 in a fixed order: block b sums the
// contiguous chunk b of the cells, then one block sums the partials in order.
constexpr int kVolBlocks = kSMs * 4;
constexpr int kVolThreads = 256;

__global__ void k_volume_partial(const double* __restrict__ H, long long n, double dA,
                                 double* __restrict__ part) {
  long long chunk = (n + gridDim.x - 1) / gridDim.x;
  long long lo = blockIdx.x * chunk, hi = lo + chunk < n ? lo + chunk : n;
  double v = 0.0, a = 0.0;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double h = H[i];
    v += h * dA;
    if (h > 0.01) a += dA;
  }
  __shared__ double sv[kVolThreads], sa[kVolThreads];
  sv[threadIdx.x] = v;
  sa[threadIdx.x] = a;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sv[threadIdx.x] += sv[threadIdx.x + s];
      sa[threadIdx.x] += sa[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sv[0];
    part[2 * blockIdx.x + 1] = sa[0];
  }
}

__global__ void k_volume_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  __shared__ double sv[kVolThreads], sa[kVolThreads];
  double v = 0.0, a = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    v += part[2 * b];
    a += part[2 * b + 1];
  }
  sv[threadIdx.x] = v;
  sa[threadIdx.x] = a;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sv[threadIdx.x] += sv[threadIdx.x + s];
      sa[threadIdx.x] += sa[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sv[0];
    out[1] = sa[0];
  }
}

// ---------------------------------------------- point boundaries, sorted
// Keys (cell << 32 | file position) sort the boundaries by cell and keep file
// order inside a cell.  An index off the grid gets the key ~0 (sorted last,
// skipped) and raises the error flag.
__global__ void k_point_keys(const int* __restrict__ idx, int n, int ncells,
                             unsigned long long* __restrict__ keys, int* __restrict__ err) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    int c = idx[k];
    if (c < 0 || c >= ncells) {
      keys[k] = ~0ULL;
      atomicOr(err, 1);
    } else {
      keys[k] = ((unsigned long long)(unsigned)c << 32) | (unsigned)k;
    }
  }
}

// Single-block bitonic sort of up to 4096 keys in shared memory.
constexpr int kSmallSort = 4096;
__global__ void k_sort_small(unsigned long long* __restrict__ keys, int n) {
  __shared__ unsigned long long s[kSmallSort];
  int m = 1;
  while (m < n) m <<= 1;
  for (int k = threadIdx.x; k < m; k += blockDim.x) s[k] = k < n ? keys[k] : ~0ULL;
  __syncthreads();
  for (int size = 2; size <= m; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = threadIdx.x; k < m; k += blockDim.x) {
        int p = k ^ stride;
        if (p > k) {
          bool up = (k & size) == 0;
          unsigned long long a = s[k], b = s[p];
          if ((a > b) == up) {
            s[k] = b;
            s[p] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int k = threadIdx.x; k < n; k += blockDim.x) keys[k] = s[k];
}

// src/main.cpp:256-260 in file order per cell: one thread per distinct cell.
__global__ void k_apply_sources(double* __restrict__ H, const unsigned long long* __restrict__ keys,
                                const double* __restrict__ ps_flow, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    unsigned long long key = keys[k];
    if (key == ~0ULL) continue;
    unsigned cell = (unsigned)(key >> 32);
    if (k > 0 && (unsigned)(keys[k - 1] >> 32) == cell) continue;  // not the segment head
    double h = H[cell];
    for (int m = k; m < n && keys[m] != ~0ULL && (unsigned)(keys[m] >> 32) == cell; m++) {
      h += ps_flow[(unsigned)(keys[m] & 0xffffffffu)];
      if (h < 0.0) h = 0.0;
    }
    H[cell] = h;
  }
}

// src/kernels.cpp:261-274 with the last effective boundary of a cell winning.
__global__ void k_apply_point_bcs(double* __restrict__ H, const unsigned long long* __restrict__ keys,
                                  const int* __restrict__ type, const double* __restrict__ value,
                                  int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    unsigned long long key = keys[k];
    if (key == ~0ULL) continue;
    unsigned cell = (unsigned)(key >> 32);
    if (k > 0 && (unsigned)(keys[k - 1] >> 32) == cell) continue;
    bool write = false;
    double v = 0.0;
    for (int m = k; m < n && keys[m] != ~0ULL && (unsigned)(keys[m] >> 32) == cell; m++) {
      unsigned b = (unsigned)(keys[m] & 0xffffffffu);
      int t = type[b];
      if (t == 1) {
        write = true;
        v = 0.0;
      } else if (t == 2 || t == 3) {
        write = true;
        v = value[b];
      }
    }
    if (write) H[cell] = v;
  }
}

// Sorts the point keys into scratch and returns the sorted array.
int sort_point_keys(const int* idx, int n, int ncells, cudaStream_t st, Scratch** sc_out,
                    unsigned long long** sorted_out, int** err_out) {
  size_t cub_bytes = 0;
  if (n > kSmallSort) {
    cub::DeviceRadixSort::SortKeys(nullptr, cub_bytes, (unsigned long long*)nullptr,
                                   (unsigned long long*)nullptr, n, 0, 64, st);
  }
  size_t keys_bytes = ((size_t)n * 8 + 255) & ~(size_t)255;
  size_t need = 256 + 2 * keys_bytes + cub_bytes;
  Scratch* sc = nullptr;
  AF_TRY(scratch_get(need, &sc));
  char* base = (char*)sc->dev;
  int* err = (int*)base;
  unsigned long long* k0 = (unsigned long long*)(base + 256);
  unsigned long long* k1 = (unsigned long long*)(base + 256 + keys_bytes);
  void* tmp = base + 256 + 2 * keys_bytes;
  AF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  k_point_keys<<<grid_for(n, 256), 256, 0, st>>>(idx, n, ncells, k0, err);
  AF_CUDA(cudaGetLastError());
  unsigned long long* sorted = k0;
  if (n > kSmallSort) {
    AF_CUDA(cub::DeviceRadixSort::SortKeys(tmp, cub_bytes, k0, k1, n, 0, 64, st));
    sorted = k1;
  } else if (n > 1) {
    k_sort_small<<<1, 1024, 0, st>>>(k0, n);
    AF_CUDA(cudaGetLastError());
  }
  *sc_out = sc;
  *sorted_out = sorted;
  *err_out = err;
  return AF_OK;
}

int finish(cudaStream_t st) {
  AF_CUDA(cudaGetLastError());
  AF_CUDA(cudaStreamSynchronize(st));
  return AF_OK;
}

}  // namespace af

using namespace af;

extern "C" {

const char* af_strerror(int code) {
  switch (code) {
    case AF_OK: return "ok";
    case AF_EINVAL: return "invalid argument";
    case AF_ERANGE: return "index or size out of range";
    case AF_ECUDA: return "CUDA error";
    case AF_ENOMEM: return "out of memory";
    case AF_EIO: return "input file missing or malformed";
    case AF_ESTATE: return "bad device state";
    default: return "unknown error";
  }
}

const char* af_last_cuda_error(void) { return af::g_last_cuda_error; }

int af_version(void) { return 10000; }

int af_update_qs(const double* Qx, const double* Qy, double* Qxold, double* Qyold, int xsz,
                 int ysz, double dx, void* stream) {
  if (xsz < 0 || ysz < 0) return AF_EINVAL;
  if (!face_count_ok(xsz, ysz)) return AF_ERANGE;
  if (!Qx || !Qy || !Qxold || !Qyold) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  long long f = (long long)(xsz + 1) * (ysz + 1);
  double dxinv = 1.0 / dx;
  k_update_qs<<<grid_for(f, 256), 256, 0, st>>>(Qx, Qy, Qxold, Qyold, f, dxinv);
  return finish(st);
}

int af_floodplain_q(const double* H, const double* DEM, double* Qx, double* Qy,
                    const double* Qxold, const double* Qyold, int xsz, int ysz, double dx,
                    double dy, double FPn, double DepthThresh, double MaxHflow, double dhlin,
                    double* Tstep, double Qlimfact, double dA, double cfl, double g,
                    double InitTstep, double theta, double nodata, void* stream) {
  (void)dy; (void)dhlin; (void)Qlimfact; (void)dA;
  if (xsz < 0 || ysz < 0 || !Tstep) return AF_EINVAL;
  if (!face_count_ok(xsz, ysz)) return AF_ERANGE;
  long long n = (long long)xsz * ysz;
  if (n > 0 && (!H || !DEM || !Qx || !Qy || !Qxold || !Qyold)) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  std::lock_guard<std::mutex> lk(scratch_lock());
  Scratch* sc = nullptr;
  AF_TRY(scratch_get(64, &sc));
  unsigned long long* acc = (unsigned long long*)sc->dev;
  double Hmax = -DBL_MAX;
  if (n > 0) {
    k_set_u64<<<1, 1, 0, st>>>(acc, ord_encode(-DBL_MAX));
    k_hmax<<<grid_for(n, 256), 256, 0, st>>>(H, DEM, n, nodata, acc);
    AF_CUDA(cudaGetLastError());
    AF_CUDA(cudaMemcpyAsync(sc->pinned, acc, 8, cudaMemcpyDeviceToHost, st));
    AF_CUDA(cudaStreamSynchronize(st));
    Hmax = ord_decode(*(unsigned long long*)sc->pinned);
  }
  double dt;  // src/kernels.cpp:36-43
  if (Hmax > DepthThresh) dt = cfl * dx / sqrt(g * Hmax);
  else dt = InitTstep;
  *Tstep = dt;
  if (xsz > 1 && ysz > 0) {
    dim3 b(32, 8), gq((xsz - 1 + 31) / 32, (ysz + 7) / 8);
    k_qx<<<gq, b, 0, st>>>(H, DEM, Qx, Qxold, Qyold, xsz, ysz, dx, FPn, DepthThresh, MaxHflow,
                           dt, g, theta, nodata);
  }
  if (xsz > 0 && ysz > 1) {
    dim3 b(32, 8), gq((xsz + 31) / 32, (ysz - 1 + 7) / 8);
    k_qy<<<gq, b, 0, st>>>(H, DEM, Qy, Qxold, Qyold, xsz, ysz, dx, FPn, DepthThresh, MaxHflow,
                           dt, g, theta, nodata);
  }
  return finish(st);
}

int af_bcs(double* Qx, double* Qy, const double* H, const double* DEM, int xsz, int ysz,
           double dx, double g, double dt, double nodata, int west_free, int east_free,
           int north_free, int south_free, void* stream) {
  (void)dt;
  if (xsz < 0 || ysz < 0) return AF_EINVAL;
  if (!face_count_ok(xsz, ysz)) return AF_ERANGE;
  if (!Qx || !Qy) return AF_EINVAL;
  if ((west_free || east_free || north_free || south_free) && (long long)xsz * ysz > 0 &&
      (!H || !DEM))
    return AF_EINVAL;
  if (west_free && xsz == 1 && ysz > 0) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  int len = (xsz > ysz ? xsz : ysz) + 1;
  dim3 g2((len + 255) / 256, 4);
  k_bcs<<<g2, 256, 0, st>>>(Qx, Qy, H, DEM, xsz, ysz, dx, g, nodata, west_free, east_free,
                            north_free, south_free);
  return finish(st);
}

int af_apply_point_bcs(double* H, const int* bc_idx, const int* bc_type, const double* bc_value,
                       int num_bcs, int ncols, double dx, double dA, double Tstep, int ncells,
                       void* stream) {
  (void)ncols; (void)dx; (void)dA; (void)Tstep;
  if (num_bcs < 0 || ncells < 0) return AF_EINVAL;
  if (num_bcs == 0) return AF_OK;
  if (!H || !bc_idx || !bc_type || !bc_value) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  std::lock_guard<std::mutex> lk(scratch_lock());
  Scratch* sc;
  unsigned long long* sorted;
  int* err;
  AF_TRY(sort_point_keys(bc_idx, num_bcs, ncells, st, &sc, &sorted, &err));
  k_apply_point_bcs<<<grid_for(num_bcs, 256), 256, 0, st>>>(H, sorted, bc_type, bc_value,
                                                             num_bcs);
  AF_CUDA(cudaGetLastError());
  AF_CUDA(cudaMemcpyAsync(sc->pinned, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  AF_TRY(finish(st));
  return *(int*)sc->pinned ? AF_ERANGE : AF_OK;
}

int af_update_h(double* H, const double* Qx, const double* Qy, int xsz, int ysz, double dA,
                double Tstep, void* stream) {
  if (xsz < 0 || ysz < 0) return AF_EINVAL;
  if (!face_count_ok(xsz, ysz)) return AF_ERANGE;
  if ((long long)xsz * ysz == 0) return AF_OK;
  if (!H || !Qx || !Qy) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  dim3 b(32, 8), g2((xsz + 31) / 32, (ysz + 7) / 8);
  k_update_h<<<g2, b, 0, st>>>(H, Qx, Qy, xsz, ysz, dA, Tstep);
  return finish(st);
}

int af_compute_velocity(double* Vx, double* Vy, const double* H, const double* DEM,
                        const double* Qx, const double* Qy, int xsz, int ysz, double dx,
                        double nodata, void* stream) {
  if (xsz < 0 || ysz < 0) return AF_EINVAL;
  if (!face_count_ok(xsz, ysz)) return AF_ERANGE;
  if ((long long)xsz * ysz == 0) return AF_OK;
  if (!Vx || !Vy || !H || !DEM || !Qx || !Qy) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  dim3 b(32, 8), g2((xsz + 31) / 32, (ysz + 7) / 8);
  k_velocity<<<g2, b, 0, st>>>(Vx, Vy, H, DEM, Qx, Qy, xsz, ysz, dx, nodata);
  return finish(st);
}

int af_rainfall(double* H, const double* DEM, int xsz, int ysz, double rain_rate, double Tstep,
                double nodata, void* stream) {
  if (xsz < 0 || ysz < 0) return AF_EINVAL;
  if (!face_count_ok(xsz, ysz)) return AF_ERANGE;
  if (rain_rate <= 0.0) return AF_OK;  // src/kernels.cpp:356
  long long n = (long long)xsz * ysz;
  if (n == 0) return AF_OK;
  if (!H || !DEM) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  double rain_depth = rain_rate * Tstep;
  k_rain<<<grid_for(n, 256), 256, 0, st>>>(H, DEM, n, rain_depth, nodata);
  return finish(st);
}

int af_add_point_sources(double* H, const int* ps_idx, const double* ps_flow, int num,
                         int ncells, void* stream) {
  if (num < 0 || ncells < 0) return AF_EINVAL;
  if (num == 0) return AF_OK;
  if (!H || !ps_idx || !ps_flow) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  std::lock_guard<std::mutex> lk(scratch_lock());
  Scratch* sc;
  unsigned long long* sorted;
  int* err;
  AF_TRY(sort_point_keys(ps_idx, num, ncells, st, &sc, &sorted, &err));
  k_apply_sources<<<grid_for(num, 256), 256, 0, st>>>(H, sorted, ps_flow, num);
  AF_CUDA(cudaGetLastError());
  AF_CUDA(cudaMemcpyAsync(sc->pinned, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  AF_TRY(finish(st));
  return *(int*)sc->pinned ? AF_ERANGE : AF_OK;
}

int af_volume_area(const double* H, int64_t n, double dA, double* vol, double* area,
                   void* stream) {
  if (n < 0 || !vol || !area) return AF_EINVAL;
  if (n == 0) {
    *vol = 0.0;
    *area = 0.0;
    return AF_OK;
  }
  if (!H) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  std::lock_guard<std::mutex> lk(scratch_lock());
  Scratch* sc = nullptr;
  AF_TRY(scratch_get(sizeof(double) * (2 * kVolBlocks + 2), &sc));
  double* part = (double*)sc->dev;
  double* out = part + 2 * kVolBlocks;
  k_volume_partial<<<kVolBlocks, kVolThreads, 0, st>>>(H, n, dA, part);
  k_volume_final<<<1, kVolThreads, 0, st>>>(part, kVolBlocks, out);
  AF_CUDA(cudaGetLastError());
  AF_CUDA(cudaMemcpyAsync(sc->pinned, out, 16, cudaMemcpyDeviceToHost, st));
  AF_TRY(finish(st));
  *vol = ((double*)sc->pinned)[0];
  *area = ((double*)sc->pinned)[1];
  return AF_OK;
}

int af_fill(double* x, int64_t n, double value, void* stream) {
  if (n < 0) return AF_EINVAL;
  if (n == 0) return AF_OK;
  if (!x) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  k_fill<<<grid_for(n, 256), 256, 0, st>>>(x, n, value);
  return finish(st);
}

int af_pow_eval(const double* x, double* out, int64_t n, double y, void* stream) {
  if (n < 0) return AF_EINVAL;
  if (n == 0) return AF_OK;
  if (!x || !out) return AF_EINVAL;
  cudaStream_t st = as_stream(stream);
  k_pow_eval<<<grid_for(n, 256), 256, 0, st>>>(x, out, n, y);
  return finish(st);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free point-source scatter.
//
// af_add_point_sources keeps its sort keys in library scratch that it grows
// with cudaMalloc.  This variant does the same work (same kernels, same
// result) with its scratch in a fixed file-scope device array instead, for
// callers that cannot have the library allocate device memory.  The array is
// part of the loaded module: every GPU that loads the library holds its
// ~33 KB until the process exits.  All calls share it, so calls whose work
// overlaps on the GPU (two streams, or two host threads) race; the error
// word is cleared by every call, and the keys are fully rewritten.
namespace af {
namespace {

constexpr int kNoAllocMaxSources = AF_NOALLOC_MAX_SOURCES;
// 32 words (256 bytes) of header -- the error flag in word 0 -- then the keys.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[32 + kNoAllocMaxSources];

// The device address of g_noalloc_scratch in the current device's context.
// In host code the symbol names a host-side shadow, not device memory, so the
// address is looked up with the device current -- on every call, not cached:
// a cached address would outlive a cudaDeviceReset (which unloads the module
// and places the array anew when it is next loaded).  The lookup neither
// allocates nor synchronises once the module is loaded on the device.
int noalloc_scratch(unsigned long long** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e);
  *out = static_cast<unsigned long long*>(p);
  return AF_OK;
}

}  // namespace
}  // namespace af

extern "C" int af_add_point_sources_noalloc(double* H, const int* ps_idx, const double* ps_flow,
                                            int num, int ncells, void* stream) {
  using namespace af;
  if (num < 0 || ncells < 0) return AF_EINVAL;
  if (num > kNoAllocMaxSources) return AF_ERANGE;  // nothing launched, H untouched
  if (num == 0) return AF_OK;
  if (!H || !ps_idx || !ps_flow) return AF_EINVAL;
  unsigned long long* scratch = nullptr;
  AF_TRY(noalloc_scratch(&scratch));
  int* err = reinterpret_cast<int*>(scratch);
  unsigned long long* keys = scratch + 32;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  AF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  k_point_keys<<<grid_for(num, 256), 256, 0, st>>>(ps_idx, num, ncells, keys, err);
  if (num > 1) k_sort_small<<<1, 1024, 0, st>>>(keys, num);
  k_apply_sources<<<grid_for(num, 256), 256, 0, st>>>(H, keys, ps_flow, num);
  AF_CUDA(cudaGetLastError());
  int host_err = 0;
  AF_CUDA(cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  AF_CUDA(cudaStreamSynchronize(st));
  return host_err ? AF_ERANGE : AF_OK;
}
