// af_simcore.cuh -- pieces shared by the single-grid simulation (af_sim.cu)
// and the batch engine (af_batch.cu): the padded field layout, the forcing
// and special-cell tables a grid's step reads, and the small kernels around
// the step (initial Hmax, velocity, volume).
//
// Padded layout of one grid in HBM (per precision T, N = 16 bytes/sizeof(T)):
//   every array has a front and back guard of kGuard elements and rows of
//   pitch P, P >= nsx*30N + N rounded up to 32 elements, so every 16-byte
//   lane vector of every strip (halo lanes included) is inside the
//   allocation and aligned;
//   H[2], DEM: ny rows of cells (column i = cell i)
//   Qx[2]:     ny rows of x-faces (column i = west face of cell i, i <= nx)
//   Qy[2]:     ny+1 rows of y-faces (row j = north face of row j)
// Padding is zero and never read into an owned result.
#pragma once

#include <vector>

#include "af_step.cuh"

namespace af {

constexpr int kGuard = 64;

// Row pitch (elements) of a grid nx wide cut into strips of 30*N columns.
inline int strips_x(int nx, int N) { return (nx + 30 * N - 1) / (30 * N); }
inline int row_pitch(int nx, int N) {
  const int P = strips_x(nx, N) * 30 * N + N;
  return (P + 31) / 32 * 32;
}
// Elements of a cell field and of the Qy field, guards included.
inline size_t cell_elems(int ny, int P) { return (size_t)kGuard * 2 + (size_t)ny * P; }
inline size_t qy_elems(int ny, int P) { return (size_t)kGuard * 2 + (size_t)(ny + 1) * P; }

inline bool non_decreasing(const double* t, int n) {
  for (int i = 0; i + 1 < n; i++)
    if (!(t[i] <= t[i + 1])) return false;
  for (int i = 0; i < n; i++)
    if (t[i] != t[i]) return false;
  return true;
}

// The first mass-report time after t (src/main.cpp:200, advanced as :303 does).
inline double first_mass_after(double t, double mass_int) {
  if (!(mass_int > 0.0)) return 0.0;
  double nm = mass_int;
  while (nm <= t) nm += mass_int;
  return nm;
}

// Host copies of everything a grid's step reads besides its fields: point
// sources stably sorted by cell (file order kept within a cell), the point
// depth BCs in file order, rain, and the special cells of every strip.
struct HostTables {
  std::vector<int> src_type, src_off;
  std::vector<double> src_value, src_times, src_vals;
  std::vector<unsigned char> src_sorted;
  std::vector<int> bc_type, bc_off;
  std::vector<double> bc_value, bc_times, bc_vals;
  std::vector<unsigned char> bc_sorted;
  std::vector<double> rain_times, rain_rates;
  int rain_sorted = 1;
  std::vector<int> spec_off;  // CSR over strip id = sy*nsx + sx
  std::vector<SpecCell> spec;
};

// Checks the case and forcing (AF_EINVAL / AF_ERANGE as af_sim_create
// documents) and builds the tables for strips of `own` columns x R rows.
int check_case(const af_case_desc* c, const af_forcing_desc* f);
void build_tables(const af_case_desc* c, const af_forcing_desc* f, int own, int R, int nsx,
                  int nsy, HostTables& t);

// ------------------------------------------------------------- kernels
template <typename T>
__global__ void k_hmax_int(const T* __restrict__ H, const T* __restrict__ Z, int nx, int ny,
                           int P, double nodata, unsigned long long* acc) {
  double m = -DBL_MAX;
  const T nd = T(nodata);
  long long n = (long long)nx * ny;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    long long j = k / nx, i = k - j * nx;
    double h = (double)H[j * P + i];
    if (Z[j * P + i] != nd && h > m) m = h;
  }
  m = warp_maxd(m);
  if ((threadIdx.x & 31) == 0 && m > -DBL_MAX) atomicMax(acc, ord_encode(m));
}

// Sets *flag when some cell of the stored DEM (state precision) equals nodata.
template <typename T>
__global__ void k_any_nodata(const T* __restrict__ Z, int nx, int ny, int P, double nodata,
                             int* flag) {
  const T nd = T(nodata);
  const long long n = (long long)nx * ny;
  bool hit = false;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const long long j = k / nx, i = k - j * nx;
    hit |= Z[j * P + i] == nd;
  }
  if (__any_sync(0xffffffffu, hit) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

static __global__ void k_ctl_fold_hmax(SimCtl* ctl) {
  ctl->hmax = ord_decode(ctl->hmax_acc);
  ctl->hmax_acc = ord_encode(-DBL_MAX);
}

// ComputeVelocity_GPU (src/kernels.cpp:293-351) on the padded layout, rows
// j0..j1-1, into dense FP64 outputs.
template <typename T>
__global__ void k_velocity_int(const T* __restrict__ H, const T* __restrict__ Z,
                               const T* __restrict__ Qx, const T* __restrict__ Qy, int nx,
                               int j0, int j1, int P, double dx, double nodata,
                               double* __restrict__ Vx, double* __restrict__ Vy) {
  long long n = (long long)nx * (j1 - j0);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    int jr = (int)(k / nx), i = (int)(k - (long long)jr * nx);
    long long r = (long long)(j0 + jr) * P;
    double z = (double)Z[r + i], h = (double)H[r + i];
    if (z == (double)T(nodata) || h < 0.001) {
      Vx[k] = 0.0;
      Vy[k] = 0.0;
      continue;
    }
    double hflow = h;
    if (hflow < 0.001) hflow = 0.001;
    double ql = (double)Qx[r + i], qr = (double)Qx[r + i + 1];
    double vl = (fabs(ql) > 1e-10) ? ql / dx / hflow : 0.0;
    double vr = (fabs(qr) > 1e-10) ? qr / dx / hflow : 0.0;
    Vx[k] = (fabs(vl) > fabs(vr)) ? vl : vr;
    double qt = (double)Qy[r + i], qb = (double)Qy[r + P + i];
    double vt = (fabs(qt) > 1e-10) ? qt / dx / hflow : 0.0;
    double vb = (fabs(qb) > 1e-10) ? qb / dx / hflow : 0.0;
    Vy[k] = (fabs(vt) > fabs(vb)) ? vt : vb;
  }
}

// Volume and flooded area of the state (src/main.cpp:293-298), fixed order.
template <typename T>
__global__ void k_volume_int(const T* __restrict__ H, int nx, int ny, int P, double dA,
                             double* __restrict__ part) {
  long long n = (long long)nx * ny;
  long long chunk = (n + gridDim.x - 1) / gridDim.x;
  long long lo = blockIdx.x * chunk, hi = min(lo + chunk, n);
  double s = 0.0, c = 0.0, a = 0.0;
  for (long long k = lo + threadIdx.x; k < hi; k += blockDim.x) {
    long long j = k / nx, i = k - j * nx;
    double h = (double)H[j * P + i];
    kahan_add(s, c, h * dA);
    if (h > 0.01) a += dA;
  }
  __shared__ double ss[256], sc[256], sa[256];
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  sa[threadIdx.x] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0.0, C = 0.0, A = 0.0;
    for (int k = 0; k < (int)blockDim.x; k++) {
      kahan_add(S, C, ss[k]);
      C += sc[k];
      A += sa[k];
    }
    part[3 * blockIdx.x] = S;
    part[3 * blockIdx.x + 1] = C;
    part[3 * blockIdx.x + 2] = A;
  }
}

// Dense FP64 rows <-> a padded FP32 field (pitch P), converted on the device:
// transfers of FP32 state move the caller's FP64 values through a device
// staging buffer in chunks, with no per-element host work.
constexpr size_t kStageBytes = 64u << 20;

static __global__ void k_pad_from_f64(const double* __restrict__ src, int rows, int width,
                               float* __restrict__ dst, int P) {
  const long long n = (long long)rows * width;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const long long j = k / width, i = k - j * width;
    dst[j * P + i] = (float)src[k];
  }
}
static __global__ void k_dense_to_f64(const float* __restrict__ src, int P, int rows, int width,
                               double* __restrict__ dst) {
  const long long n = (long long)rows * width;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const long long j = k / width, i = k - j * width;
    dst[k] = (double)src[j * P + i];
  }
}

}  // namespace af
