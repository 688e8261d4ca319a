// af_sim.cu -- the simulation layer: device-resident state, forcing tables,
// special-cell lists, and the CUDA graph that runs the time loop of one grid.
// The padded field layout is described in af_simcore.cuh.
//
// The time loop (src/main.cpp:227 `while (t < sim_time)`) is one graph
// launch: a begin kernel sets the stop condition, then a conditional WHILE
// node re-runs the step kernel until its last block clears the condition.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include <sys/stat.h>

#include "af_output.h"
#include "af_simcore.cuh"
#include "af_xfer.h"

namespace af {

constexpr int kMassCap = 1 << 16;

struct DevBuf {
  void* p = nullptr;
  bool own = true;  // false: a view into another buffer's allocation
  ~DevBuf() {
    if (p && own) cudaFree(p);
  }
};

template <typename V>
static int upload(DevBuf& b, const std::vector<V>& v, cudaStream_t st) {
  size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(V);
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cuda_fail(e);
    return AF_ENOMEM;
  }
  if (!v.empty()) AF_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(V),
                                          cudaMemcpyHostToDevice, st));
  return AF_OK;
}

int check_case(const af_case_desc* c, const af_forcing_desc* f) {
  if (!c || !f) return AF_EINVAL;
  if (c->nx < 2 || c->ny < 2) return AF_EINVAL;
  if (!(c->dx > 0.0) || c->theta != 1.0) return AF_EINVAL;
  if ((long long)(c->nx + 1) * (c->ny + 1) > 0x7FFFFFFFLL) return AF_ERANGE;
  if (f->n_flow < 0 || f->n_other < 0 || f->n_rain < 0) return AF_EINVAL;
  const long long ncell = (long long)c->nx * c->ny;
  for (int k = 0; k < f->n_flow; k++)
    if (f->flow_idx[k] < 0 || f->flow_idx[k] >= ncell) return AF_ERANGE;
  for (int k = 0; k < f->n_other; k++)
    if (f->other_idx[k] < 0 || f->other_idx[k] >= ncell) return AF_ERANGE;
  return AF_OK;
}

void build_tables(const af_case_desc* c, const af_forcing_desc* f, int own, int R, int nsx,
                  int nsy, HostTables& t) {
  const int nx = c->nx;
  // ---- point sources, stably sorted by cell (file order kept per cell)
  std::vector<int> order(f->n_flow);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return f->flow_idx[a] < f->flow_idx[b]; });
  t.src_off.assign(1, 0);
  for (int k : order) {
    t.src_type.push_back(f->flow_type[k]);
    t.src_value.push_back(f->flow_value[k]);
    int n = 0;
    if (f->flow_type[k] == AF_BC_QVAR) {
      int o = f->flow_off[k];
      n = f->flow_off[k + 1] - o;
      t.src_times.insert(t.src_times.end(), f->flow_times + o, f->flow_times + o + n);
      t.src_vals.insert(t.src_vals.end(), f->flow_vals + o, f->flow_vals + o + n);
      t.src_sorted.push_back(non_decreasing(f->flow_times + o, n) ? 1 : 0);
    } else {
      t.src_sorted.push_back(1);
    }
    t.src_off.push_back(t.src_off.back() + n);
  }
  // ---- point depth BCs: the last effective one per cell wins (file order)
  t.bc_type.resize(f->n_other);
  t.bc_off.assign(f->n_other + 1, 0);
  t.bc_value.resize(f->n_other);
  t.bc_sorted.resize(f->n_other);
  for (int k = 0; k < f->n_other; k++) {
    t.bc_type[k] = f->other_type[k];
    t.bc_value[k] = f->other_value[k];
    int n = 0;
    if (t.bc_type[k] == AF_BC_HVAR) {
      int o = f->other_off[k];
      n = f->other_off[k + 1] - o;
      t.bc_times.insert(t.bc_times.end(), f->other_times + o, f->other_times + o + n);
      t.bc_vals.insert(t.bc_vals.end(), f->other_vals + o, f->other_vals + o + n);
    }
    t.bc_off[k + 1] = t.bc_off[k] + n;
    t.bc_sorted[k] = non_decreasing(t.bc_times.data() + t.bc_off[k], n) ? 1 : 0;
  }
  // ---- special cells
  struct Ent {
    long long strip;
    SpecCell e;
  };
  std::vector<Ent> ents;
  {
    size_t k = 0;
    std::vector<std::pair<int, int>> last_bc;  // (cell, bc)
    for (int b = 0; b < f->n_other; b++)
      if (t.bc_type[b] == 1 || t.bc_type[b] == 2 || t.bc_type[b] == 3)
        last_bc.push_back({f->other_idx[b], b});
    std::stable_sort(last_bc.begin(), last_bc.end(),
                     [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
                       return a.first < b.first;
                     });
    std::vector<std::pair<int, int>> bc_of;  // cell -> last bc
    for (size_t q = 0; q < last_bc.size(); q++)
      if (q + 1 == last_bc.size() || last_bc[q + 1].first != last_bc[q].first)
        bc_of.push_back(last_bc[q]);
    size_t qb = 0;
    auto emit = [&](int cell, int s0, int s1, int bc) {
      SpecCell e{};
      e.row = cell / nx;
      e.col = cell % nx;
      e.s0 = s0;
      e.s1 = s1;
      e.bc = bc;
      int sx = e.col / own, sy = e.row / R;
      long long strip = (long long)sx * nsy + sy;  // column-major: order independent of R
      ents.push_back({strip, e});
    };
    // merge the sorted source cells with the sorted bc cells
    while (k < order.size() || qb < bc_of.size()) {
      int cs = k < order.size() ? f->flow_idx[order[k]] : 0x7FFFFFFF;
      int cbc = qb < bc_of.size() ? bc_of[qb].first : 0x7FFFFFFF;
      int cell = std::min(cs, cbc);
      int s0 = (int)k;
      while (k < order.size() && f->flow_idx[order[k]] == cell) k++;
      int bc = -1;
      if (cbc == cell) {
        bc = bc_of[qb].second;
        qb++;
      }
      emit(cell, s0, (int)k, bc);
    }
  }
  // Sorted by (strip, row, col); with column-major strip ids this is the
  // order (column strip, row, col) whatever the strip height.
  std::stable_sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) {
    if (a.strip != b.strip) return a.strip < b.strip;
    if (a.e.row != b.e.row) return a.e.row < b.e.row;
    return a.e.col < b.e.col;
  });
  const long long nstrips = (long long)nsx * nsy;
  t.spec_off.assign(nstrips + 1, 0);
  t.spec.clear();
  for (auto& e : ents) {
    t.spec_off[e.strip + 1]++;
    t.spec.push_back(e.e);
  }
  for (long long q = 0; q < nstrips; q++) t.spec_off[q + 1] += t.spec_off[q];
  t.rain_times.assign(f->rain_times, f->rain_times + f->n_rain);
  t.rain_rates.assign(f->rain_rates, f->rain_rates + f->n_rain);
  t.rain_sorted = non_decreasing(t.rain_times.data(), f->n_rain) ? 1 : 0;
}

// Sets the stop condition of one launch: the loop runs while t < t_stop and
// fewer than max_steps steps have run in this launch.
__global__ void k_begin(SimCtl* ctl, double t_stop, long long max_steps,
                        cudaGraphConditionalHandle cond, int use_cond) {
  ctl->t_stop = t_stop;
  long long s = ctl->step;
  ctl->step_stop = (max_steps > (long long)0x3FFFFFFFFFFFFFFFLL - s) ? 0x3FFFFFFFFFFFFFFFLL
                                                                      : s + max_steps;
  // A simulation whose state went bad stays stopped (no further steps).
  int done = !(ctl->t < t_stop) || max_steps <= 0 || ctl->status != 0;
  ctl->done = done;
  ctl->arrive = 0u;
  if (use_cond) cudaGraphSetConditional(cond, done ? 0u : 1u);
}

// Snapshot of the state for the file outputs: H and, when asked, the
// velocity of ComputeVelocity_GPU (src/kernels.cpp:293-351), as dense FP64
// fields in the reference layout.
template <typename T>
__global__ void k_snapshot(const T* __restrict__ H, const T* __restrict__ Z,
                           const T* __restrict__ Qx, const T* __restrict__ Qy, int nx, int ny,
                           int P, double dx, double nodata, double* __restrict__ oH,
                           double* __restrict__ oVx, double* __restrict__ oVy) {
  const long long n = (long long)nx * ny;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(k / nx), i = (int)(k - (long long)j * nx);
    const long long r = (long long)j * P;
    const double h = (double)H[r + i];
    oH[k] = h;
    if (!oVx) continue;
    const double z = (double)Z[r + i];
    if (z == (double)T(nodata) || h < 0.001) {
      oVx[k] = 0.0;
      oVy[k] = 0.0;
      continue;
    }
    double hflow = h;
    if (hflow < 0.001) hflow = 0.001;
    const double ql = (double)Qx[r + i], qr = (double)Qx[r + i + 1];
    const double vl = (fabs(ql) > 1e-10) ? ql / dx / hflow : 0.0;
    const double vr = (fabs(qr) > 1e-10) ? qr / dx / hflow : 0.0;
    oVx[k] = (fabs(vl) > fabs(vr)) ? vl : vr;
    const double qt = (double)Qy[r + i], qb = (double)Qy[r + P + i];
    const double vt = (fabs(qt) > 1e-10) ? qt / dx / hflow : 0.0;
    const double vb = (fabs(qb) > 1e-10) ? qb / dx / hflow : 0.0;
    oVy[k] = (fabs(vt) > fabs(vb)) ? vt : vb;
  }
}

// Depths at the stage points (src/main.cpp:306-322); -1 = outside the grid.
template <typename T>
__global__ void k_gather(const T* __restrict__ H, int nx, int P, const int* __restrict__ idx,
                         int n, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = idx[k];
  out[k] = c < 0 ? 0.0 : (double)H[(long long)(c / nx) * P + c % nx];
}

// ----------------------------------------------------------- the object
struct Sim {
  int device = 0;
  int prec = AF_PREC_F64;
  int esize = 8, N = 2;
  cudaStream_t st = nullptr;
  af_case_desc c{};
  int P = 0, nsx = 0, nsy = 0, R = 16, WY = 4, variant = 0;
  bool face_call = false;  // FP64: the step kernel with out-of-line faces
  bool tma = true;         // the step kernel reads rows with tiled copies
  size_t cells_elems = 0, qy_elems = 0;  // field sizes (elements, guards included)
  // The fields are planes of one allocation, each qy_elems long, in the order
  // H0, DEM, Qx0, Qy0, H1, DEM (a copy), Qx1, Qy1: the four fields a step
  // reads are then planes 4*parity .. 4*parity+3 of one 3-D tensor, which
  // the step kernel's tiled copies (tensor map `fields`) read in one box.
  DevBuf planes;
  DevBuf H[2], Qx[2], Qy[2], DEM, DEM2;  // views into `planes`
  CUtensorMap fields;
  DevBuf src_type, src_value, src_off, src_times, src_vals, src_sorted;
  DevBuf bc_type, bc_value, bc_off, bc_times, bc_vals, bc_sorted;
  DevBuf rain_times, rain_rates, spec_off, spec;
  DevBuf ctl, partials, mass_series;
  SimCtl* pinned_ctl = nullptr;
  StepParams prm{};
  dim3 grid, block;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t begin_node = nullptr;
  cudaGraphConditionalHandle cond = 0;
  bool use_cond = false;
  int n_rain = 0;
  std::vector<double> rain_t, rain_r;
  uint64_t case_hash = 0;  // case parameters and forcing (checkpoint identity)

  ~Sim() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (pinned_ctl) cudaFreeHost(pinned_ctl);
    if (st) cudaStreamDestroy(st);
  }

  template <typename T>
  T* buf(DevBuf& b) const { return static_cast<T*>(b.p) + kGuard; }
};

// The step kernel of the simulation's precision, shape and face evaluation.
static const void* step_fn(const Sim& s) {
  return s.prec == AF_PREC_F64 ? step_kernel_f64(s.variant, s.face_call, s.tma)
                               : step_kernel_f32(s.variant, s.tma);
}

static int pick_shape(Sim& s) {
  const int own = 30 * s.N;
  s.nsx = (s.c.nx + own - 1) / own;
  // Launch shape: FP32 one-warp blocks, 16 per SM (120 registers); FP64 20 per
  // SM (96 registers: measured 6 % faster than 16 per SM on the 8192^2 step).
  s.variant = s.prec == AF_PREC_F64 ? 2 : 0;
  if (const char* v = getenv("AF_SIM_VARIANT")) {
    const int k = atoi(v);
    if (k >= 0 && k < kStepVariants) s.variant = k;
  }
  s.WY = kStepVariant[s.variant].wy;
  s.face_call = face_call_for(s.prec == AF_PREC_F64, (long long)s.c.nx * s.c.ny);
  s.tma = tma_for(s.prec == AF_PREC_F64, (long long)s.c.nx * s.c.ny);
  const void* fn = step_fn(s);
  int per_sm = 0, dev = 0, sms = kSMs;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * s.WY, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long slots = (long long)sms * per_sm;  // resident blocks
  auto tiles_for = [&](int R) {
    const long long nsy = (s.c.ny + R - 1) / R;
    return (long long)s.nsx * ((nsy + s.WY - 1) / s.WY);
  };
  // Rows per strip.  Large grids take 32 (measured best at 8192^2: taller
  // strips lose DRAM locality between the warps running side by side, shorter
  // ones pay their prologue row more often).  In FP32 a grid whose 32-row
  // strips fill at most two waves of the resident blocks takes the shortest
  // strips that still fit in as many waves, so every block gets the same
  // number of strips and each is as short as it can be (measured against
  // powers of two: 512^2 +21 %, 2048^2 +6 %, 4096^2 +5 %).  The FP64 step,
  // bound by its arithmetic, keeps more, shorter strips on mid-size grids
  // (measured 8-9 % faster than the two-wave rule at 2048^2 and 4096^2), and
  // on grids of up to 2^20 cells (less than one wave) two-row strips, the
  // shortest serial chain per warp (512^2: 34.7 ms for the 1442-step C1 run
  // against 50.2 ms with four rows).
  const long long cells = (long long)s.c.nx * s.c.ny;
  s.R = 32;
  if (s.prec == AF_PREC_F64) {
    if (cells <= (1LL << 20)) s.R = 2;
    else if (cells <= (1LL << 23)) s.R = 8;
    else if (cells <= (1LL << 25)) s.R = 16;
  } else if (cells < (1LL << 20)) {
    // Small FP32 grids: one-row strips, the shortest chain per warp even at
    // slightly over one wave (ms per step, one row against the two-wave rule:
    // 512^2 0.0312 / 0.0369, 724^2 0.0372 / 0.0393; at 1024^2 and above the
    // rule is as fast or faster).
    s.R = 1;
  } else {
    const long long waves = (tiles_for(32) + slots - 1) / slots;
    if (waves <= 2) {
      for (int R = 2; R < 32; R++)
        if (tiles_for(R) <= waves * slots) {
          s.R = R;
          break;
        }
    }
  }
  if (const char* r = getenv("AF_SIM_ROWS")) {  // strip height override (tuning sweeps)
    const int v = atoi(r);
    if (v >= 1 && v <= 4096) s.R = v;
  }
  s.nsy = (s.c.ny + s.R - 1) / s.R;
  // Persistent grid: as many blocks as fit on the GPU at once (a whole number
  // of blocks per SM), never more than there are tiles.
  const long long tiles = (long long)s.nsx * ((s.nsy + s.WY - 1) / s.WY);
  s.grid = dim3((unsigned)(tiles < slots ? tiles : slots));
  s.block = dim3(32 * s.WY);
  return AF_OK;
}

// The tensor map of the field planes (see encode_field_planes).
static int encode_fields(Sim& s) {
  void* origin = static_cast<char*>(s.planes.p) + (size_t)kGuard * s.esize;
  return encode_field_planes(&s.fields, origin, s.esize, s.c.nx, s.c.ny, s.P,
                             s.qy_elems * s.esize);
}

static int alloc_field(DevBuf& b, size_t elems, int esize) {
  cudaError_t e = cudaMalloc(&b.p, elems * esize);
  if (e != cudaSuccess) {
    cuda_fail(e);
    return AF_ENOMEM;
  }
  return AF_OK;
}

// Copies a host FP64 field with `rows` x `width` entries and host pitch
// `hpitch` into the padded device field (converted to the sim precision).
// Field transfers between the caller's FP64 host arrays (rows of `width`
// values at host pitch `hpitch`) and a padded device field.  FP64 fields are
// one 2-D copy.  FP32 fields go through a dense FP64 device staging buffer in
// chunks of rows, converted by a kernel on the device, so the host does no
// per-element work (and pinned host arrays move at full link bandwidth).
static int put_field(Sim& s, DevBuf& b, const double* src, int rows, int width, size_t hpitch) {
  char* dst = static_cast<char*>(b.p) + (size_t)kGuard * s.esize;
  if (s.prec == AF_PREC_F64) {
    AF_CUDA(copy2d_h2d(dst, (size_t)s.P * 8, src, hpitch * 8, (size_t)width * 8, rows, s.st));
    AF_CUDA(cudaStreamSynchronize(s.st));
    return AF_OK;
  }
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>(rows, kStageBytes / (8 * (size_t)width)));
  DevBuf stage;
  AF_TRY(alloc_field(stage, (size_t)chunk * width, 8));
  for (int j = 0; j < rows; j += chunk) {
    const int n = std::min(chunk, rows - j);
    AF_CUDA(copy2d_h2d(stage.p, (size_t)width * 8, src + (size_t)j * hpitch, hpitch * 8,
                       (size_t)width * 8, n, s.st));
    k_pad_from_f64<<<grid_for((long long)n * width, 256, 8), 256, 0, s.st>>>(
        static_cast<const double*>(stage.p), n, width,
        reinterpret_cast<float*>(dst) + (size_t)j * s.P, s.P);
    AF_CUDA(cudaGetLastError());
  }
  AF_CUDA(cudaStreamSynchronize(s.st));
  return AF_OK;
}

static int get_field(Sim& s, DevBuf& b, double* dst, int rows, int width, size_t hpitch) {
  const char* src = static_cast<const char*>(b.p) + (size_t)kGuard * s.esize;
  if (s.prec == AF_PREC_F64) {
    AF_CUDA(copy2d_d2h(dst, hpitch * 8, src, (size_t)s.P * 8, (size_t)width * 8, rows, s.st));
    AF_CUDA(cudaStreamSynchronize(s.st));
    return AF_OK;
  }
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>(rows, kStageBytes / (8 * (size_t)width)));
  DevBuf stage;
  AF_TRY(alloc_field(stage, (size_t)chunk * width, 8));
  for (int j = 0; j < rows; j += chunk) {
    const int n = std::min(chunk, rows - j);
    k_dense_to_f64<<<grid_for((long long)n * width, 256, 8), 256, 0, s.st>>>(
        reinterpret_cast<const float*>(src) + (size_t)j * s.P, s.P, n, width,
        static_cast<double*>(stage.p));
    AF_CUDA(cudaGetLastError());
    AF_CUDA(copy2d_d2h(dst + (size_t)j * hpitch, hpitch * 8, stage.p, (size_t)width * 8,
                       (size_t)width * 8, n, s.st));
  }
  AF_CUDA(cudaStreamSynchronize(s.st));
  return AF_OK;
}

static int refresh_hmax(Sim& s, int parity) {
  SimCtl* ctl = static_cast<SimCtl*>(s.ctl.p);
  unsigned grid = grid_for((long long)s.c.nx * s.c.ny, 256, 8);
  if (s.prec == AF_PREC_F64)
    k_hmax_int<double><<<grid, 256, 0, s.st>>>(s.buf<double>(s.H[parity]), s.buf<double>(s.DEM),
                                               s.c.nx, s.c.ny, s.P, s.c.nodata, &ctl->hmax_acc);
  else
    k_hmax_int<float><<<grid, 256, 0, s.st>>>(s.buf<float>(s.H[parity]), s.buf<float>(s.DEM),
                                              s.c.nx, s.c.ny, s.P, s.c.nodata, &ctl->hmax_acc);
  k_ctl_fold_hmax<<<1, 1, 0, s.st>>>(ctl);
  AF_CUDA(cudaGetLastError());
  return AF_OK;
}

// Whether the stored DEM has a nodata cell (one word of the partials buffer,
// which holds nothing between launches, as the flag).
static int any_nodata(Sim& s, int* out) {
  int* flag = static_cast<int*>(s.partials.p);
  AF_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s.st));
  const unsigned grid = grid_for((long long)s.c.nx * s.c.ny, 256, 8);
  if (s.prec == AF_PREC_F64)
    k_any_nodata<double><<<grid, 256, 0, s.st>>>(s.buf<double>(s.DEM), s.c.nx, s.c.ny, s.P,
                                                 s.c.nodata, flag);
  else
    k_any_nodata<float><<<grid, 256, 0, s.st>>>(s.buf<float>(s.DEM), s.c.nx, s.c.ny, s.P,
                                                s.c.nodata, flag);
  AF_CUDA(cudaGetLastError());
  int h = 0;
  AF_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s.st));
  AF_CUDA(cudaStreamSynchronize(s.st));
  *out = h;
  return AF_OK;
}

static int read_ctl(Sim& s) {
  AF_CUDA(cudaMemcpyAsync(s.pinned_ctl, s.ctl.p, sizeof(SimCtl), cudaMemcpyDeviceToHost, s.st));
  AF_CUDA(cudaStreamSynchronize(s.st));
  return AF_OK;
}

static int write_ctl(Sim& s) {
  AF_CUDA(cudaMemcpyAsync(s.ctl.p, s.pinned_ctl, sizeof(SimCtl), cudaMemcpyHostToDevice, s.st));
  AF_CUDA(cudaStreamSynchronize(s.st));
  return AF_OK;
}

static int build_graph(Sim& s) {
  // AF_SIM_DIRECT_LAUNCH=1 launches the same step kernel from the host in
  // batches instead of through the conditional graph: profilers cannot see
  // kernel nodes inside graphs that contain conditional nodes.
  const char* direct = getenv("AF_SIM_DIRECT_LAUNCH");
  if (direct && direct[0] && direct[0] != '0') return AF_OK;
  AF_CUDA(cudaGraphCreate(&s.graph, 0));
  SimCtl* ctl = static_cast<SimCtl*>(s.ctl.p);
  s.use_cond = cudaGraphConditionalHandleCreate(&s.cond, s.graph, 0, 0) == cudaSuccess;
  if (!s.use_cond) {
    cudaGetLastError();
    cudaGraphDestroy(s.graph);
    s.graph = nullptr;
    return AF_OK;  // fall back to host-driven launches
  }
  s.prm.cond = s.cond;
  s.prm.use_cond = 1;
  double t_stop = 0.0;
  long long max_steps = 0;
  int use = 1;
  void* bargs[] = {&ctl, &t_stop, &max_steps, &s.cond, &use};
  cudaKernelNodeParams kb{};
  kb.func = (void*)&k_begin;
  kb.gridDim = dim3(1);
  kb.blockDim = dim3(1);
  kb.kernelParams = bargs;
  AF_CUDA(cudaGraphAddKernelNode(&s.begin_node, s.graph, nullptr, 0, &kb));

  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = s.cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  AF_CUDA(cudaGraphAddNode(&cnode, s.graph, &s.begin_node, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];

  // The loop body is kStepsPerIteration steps in a row: a step after the
  // one that ended the loop finds the control block done and returns at
  // once, and the loop test runs once per iteration instead of once per step.
  void* sargs[] = {&s.prm, &s.fields};
  cudaKernelNodeParams ks{};
  ks.func = const_cast<void*>(step_fn(s));
  ks.gridDim = s.grid;
  ks.blockDim = s.block;
  ks.kernelParams = sargs;
  cudaGraphNode_t prev = nullptr;
  for (int k = 0; k < kStepsPerIteration; k++) {
    cudaGraphNode_t snode;
    AF_CUDA(cudaGraphAddKernelNode(&snode, body, prev ? &prev : nullptr, prev ? 1 : 0, &ks));
    prev = snode;
  }
  AF_CUDA(cudaGraphInstantiate(&s.exec, s.graph, 0));
  return AF_OK;
}

// Identity of a case for checkpoints: a 64-bit mix (splitmix64 finaliser)
// of every parameter and forcing value, position by position.
static inline uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
struct Hasher {
  uint64_t h = 0x6166636b70743032ULL, n = 0;
  void word(uint64_t w) { h = mix64(h ^ mix64(w + 0x9e3779b97f4a7c15ULL * ++n)); }
  void d(double v) {
    uint64_t w;
    memcpy(&w, &v, 8);
    word(w);
  }
  void i(long long v) { word((uint64_t)v); }
  template <typename T>
  void arr(const T* a, long long k) {
    i(k);
    for (long long q = 0; q < (a ? k : 0); q++) {
      if (sizeof(T) == 8) d((double)a[q]);
      else i((long long)a[q]);
    }
  }
};
static uint64_t case_hash(const af_case_desc* c, const af_forcing_desc* f) {
  Hasher h;
  h.i(c->nx); h.i(c->ny);
  h.d(c->dx); h.d(c->nodata); h.d(c->fpn); h.d(c->depth_thresh); h.d(c->cfl);
  h.d(c->init_tstep); h.d(c->g); h.d(c->max_hflow); h.d(c->theta); h.d(c->mass_int);
  h.i(c->west_free); h.i(c->east_free); h.i(c->north_free); h.i(c->south_free);
  const int nf = f->n_flow, no = f->n_other;
  const long long fser = (nf > 0 && f->flow_off) ? f->flow_off[nf] : 0;
  const long long oser = (no > 0 && f->other_off) ? f->other_off[no] : 0;
  h.arr(f->flow_idx, nf); h.arr(f->flow_type, nf); h.arr(f->flow_value, nf);
  h.arr(f->flow_off, nf > 0 ? nf + 1 : 0); h.arr(f->flow_times, fser); h.arr(f->flow_vals, fser);
  h.arr(f->other_idx, no); h.arr(f->other_type, no); h.arr(f->other_value, no);
  h.arr(f->other_off, no > 0 ? no + 1 : 0); h.arr(f->other_times, oser);
  h.arr(f->other_vals, oser);
  h.arr(f->rain_times, f->n_rain); h.arr(f->rain_rates, f->n_rain);
  return h.h;
}

// Order-free hash of the stored DEM: the wrapping sum over valid cells of a
// mix of (value bits, cell index), so the result does not depend on the
// launch shape.
template <typename T>
__global__ void k_dem_hash(const T* __restrict__ Z, int nx, int ny, int P,
                           unsigned long long* out) {
  const long long n = (long long)nx * ny;
  unsigned long long acc = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(k / nx), i = (int)(k - (long long)j * nx);
    unsigned long long w;
    if (sizeof(T) == 8) w = (unsigned long long)__double_as_longlong((double)Z[(long long)j * P + i]);
    else w = (unsigned long long)__float_as_uint((float)Z[(long long)j * P + i]);
    unsigned long long x = w ^ (0x9e3779b97f4a7c15ULL * (unsigned long long)(k + 1));
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    acc += x ^ (x >> 31);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

static int create(const af_case_desc* c, const af_forcing_desc* f, const double* dem,
                  const double* h0, int precision, int device, Sim** out) {
  if (!c || !f || !dem || !out) return AF_EINVAL;
  if (precision != AF_PREC_F64 && precision != AF_PREC_F32) return AF_EINVAL;
  AF_TRY(check_case(c, f));

  std::unique_ptr<Sim> s(new Sim());
  s->device = device;
  s->prec = precision;
  s->esize = precision == AF_PREC_F64 ? 8 : 4;
  s->N = 16 / s->esize;
  s->c = *c;
  s->case_hash = case_hash(c, f);
  AF_CUDA(cudaSetDevice(device));
  AF_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  AF_CUDA(cudaMallocHost(&s->pinned_ctl, sizeof(SimCtl)));
  pick_shape(*s);
  const int own = 30 * s->N;
  const int P = row_pitch(c->nx, s->N);
  s->P = P;
  const int nx = c->nx, ny = c->ny;
  s->cells_elems = cell_elems(ny, P);
  s->qy_elems = qy_elems(ny, P);
  if (const char* e = getenv("AF_PLANE_PAD")) s->qy_elems += (size_t)atoll(e);  // EXPERIMENT
  const size_t plane_bytes = s->qy_elems * s->esize;
  AF_TRY(alloc_field(s->planes, 8 * s->qy_elems, s->esize));
  AF_CUDA(cudaMemsetAsync(s->planes.p, 0, 8 * plane_bytes, s->st));
  DevBuf* order[8] = {&s->H[0], &s->DEM, &s->Qx[0], &s->Qy[0],
                      &s->H[1], &s->DEM2, &s->Qx[1], &s->Qy[1]};
  for (int k = 0; k < 8; k++) {
    order[k]->p = static_cast<char*>(s->planes.p) + k * plane_bytes;
    order[k]->own = false;
  }
  AF_TRY(put_field(*s, s->DEM, dem, ny, nx, nx));
  AF_CUDA(cudaMemcpyAsync(s->DEM2.p, s->DEM.p, plane_bytes, cudaMemcpyDeviceToDevice, s->st));
  if (h0) AF_TRY(put_field(*s, s->H[0], h0, ny, nx, nx));
  AF_TRY(encode_fields(*s));

  HostTables tb;
  build_tables(c, f, own, s->R, s->nsx, s->nsy, tb);
  AF_TRY(upload(s->src_type, tb.src_type, s->st));
  AF_TRY(upload(s->src_value, tb.src_value, s->st));
  AF_TRY(upload(s->src_off, tb.src_off, s->st));
  AF_TRY(upload(s->src_times, tb.src_times, s->st));
  AF_TRY(upload(s->src_vals, tb.src_vals, s->st));
  AF_TRY(upload(s->src_sorted, tb.src_sorted, s->st));
  AF_TRY(upload(s->bc_type, tb.bc_type, s->st));
  AF_TRY(upload(s->bc_value, tb.bc_value, s->st));
  AF_TRY(upload(s->bc_off, tb.bc_off, s->st));
  AF_TRY(upload(s->bc_times, tb.bc_times, s->st));
  AF_TRY(upload(s->bc_vals, tb.bc_vals, s->st));
  AF_TRY(upload(s->bc_sorted, tb.bc_sorted, s->st));
  s->rain_t = tb.rain_times;
  s->rain_r = tb.rain_rates;
  s->n_rain = f->n_rain;
  AF_TRY(upload(s->rain_times, s->rain_t, s->st));
  AF_TRY(upload(s->rain_rates, s->rain_r, s->st));
  AF_TRY(upload(s->spec_off, tb.spec_off, s->st));
  AF_TRY(upload(s->spec, tb.spec, s->st));
  const size_t nblocks = (size_t)s->grid.x * s->grid.y;
  AF_TRY(alloc_field(s->partials, nblocks * 3 + 3, 8));
  AF_TRY(alloc_field(s->mass_series, (size_t)kMassCap * 3, 8));
  AF_TRY(alloc_field(s->ctl, 1, sizeof(SimCtl)));

  SimCtl& h = *s->pinned_ctl;
  memset(&h, 0, sizeof(SimCtl));
  h.t = 0.0;
  h.hmax = -DBL_MAX;
  h.rain_rate = s->n_rain > 0 ? interp_series(s->rain_t.data(), s->rain_r.data(), s->n_rain, 0.0,
                                              0.0, non_decreasing(s->rain_t.data(), s->n_rain))
                              : 0.0;
  h.next_mass = first_mass_after(0.0, c->mass_int);
  h.hmax_acc = ord_encode(-DBL_MAX);
  h.done = 1;
  h.mass_cap = kMassCap;
  AF_TRY(write_ctl(*s));
  AF_TRY(refresh_hmax(*s, 0));

  StepParams& p = s->prm;
  for (int b = 0; b < 2; b++) {
    p.H[b] = static_cast<char*>(s->H[b].p) + (size_t)kGuard * s->esize;
    p.Qx[b] = static_cast<char*>(s->Qx[b].p) + (size_t)kGuard * s->esize;
    p.Qy[b] = static_cast<char*>(s->Qy[b].p) + (size_t)kGuard * s->esize;
  }
  p.DEM = static_cast<char*>(s->DEM.p) + (size_t)kGuard * s->esize;
  p.nx = nx;
  p.ny = ny;
  p.P = P;
  p.nsx = s->nsx;
  p.nsy = s->nsy;
  p.R = s->R;
  p.dx = c->dx;
  p.dxinv = 1.0 / c->dx;  // src/kernels.cpp:8
  p.dA = c->dx * c->dx;   // src/main.cpp:115
  p.fpn = c->fpn;
  p.depth_thresh = c->depth_thresh;
  p.max_hflow = c->max_hflow;
  p.g = c->g;
  p.cfl = c->cfl;
  p.init_tstep = c->init_tstep;
  p.nodata = c->nodata;
  p.mass_int = c->mass_int;
  p.wf = c->west_free;
  p.ef = c->east_free;
  p.nf = c->north_free;
  p.sf = c->south_free;
  AF_TRY(any_nodata(*s, &p.has_nodata));
  p.src_type = (const int*)s->src_type.p;
  p.src_value = (const double*)s->src_value.p;
  p.src_off = (const int*)s->src_off.p;
  p.src_times = (const double*)s->src_times.p;
  p.src_vals = (const double*)s->src_vals.p;
  p.src_sorted = (const unsigned char*)s->src_sorted.p;
  p.bc_type = (const int*)s->bc_type.p;
  p.bc_value = (const double*)s->bc_value.p;
  p.bc_off = (const int*)s->bc_off.p;
  p.bc_times = (const double*)s->bc_times.p;
  p.bc_vals = (const double*)s->bc_vals.p;
  p.bc_sorted = (const unsigned char*)s->bc_sorted.p;
  p.rain_times = (const double*)s->rain_times.p;
  p.rain_rates = (const double*)s->rain_rates.p;
  p.n_rain = s->n_rain;
  p.rain_sorted = tb.rain_sorted;
  p.spec_off = (const int*)s->spec_off.p;
  p.spec = (const SpecCell*)s->spec.p;
  p.ctl = static_cast<SimCtl*>(s->ctl.p);
  p.partials = static_cast<double*>(s->partials.p);
  p.mass_series = static_cast<double*>(s->mass_series.p);
  p.use_cond = 0;
  AF_TRY(build_graph(*s));
  AF_CUDA(cudaStreamSynchronize(s->st));
  *out = s.release();
  return AF_OK;
}

static int launch(Sim& s, double t_stop, long long max_steps) {
  AF_CUDA(cudaSetDevice(s.device));
  SimCtl* ctl = static_cast<SimCtl*>(s.ctl.p);
  if (s.use_cond) {
    int use = 1;
    void* bargs[] = {&ctl, &t_stop, &max_steps, &s.cond, &use};
    cudaKernelNodeParams kb{};
    kb.func = (void*)&k_begin;
    kb.gridDim = dim3(1);
    kb.blockDim = dim3(1);
    kb.kernelParams = bargs;
    AF_CUDA(cudaGraphExecKernelNodeSetParams(s.exec, s.begin_node, &kb));
    AF_CUDA(cudaGraphLaunch(s.exec, s.st));
    return AF_OK;
  }
  // Host-driven fallback: launch steps in batches, checking completion.
  k_begin<<<1, 1, 0, s.st>>>(ctl, t_stop, max_steps, 0, 0);
  const void* fn = step_fn(s);
  StepParams p = s.prm;
  void* args[] = {&p, &s.fields};
  long long left = max_steps;
  while (left > 0) {
    long long batch = left < 64 ? left : 64;
    for (long long k = 0; k < batch; k++)
      AF_CUDA(cudaLaunchKernel(fn, s.grid, s.block, args, 0, s.st));
    left -= batch;
    AF_TRY(read_ctl(s));
    if (s.pinned_ctl->done) break;
  }
  return AF_OK;
}

}  // namespace af

using af::Sim;

struct af_sim {
  Sim* s;
};

extern "C" {

int af_sim_create(const af_case_desc* c, const af_forcing_desc* f, const double* dem,
                  const double* h0, int precision, int device, af_sim** out) {
  if (!out) return AF_EINVAL;
  Sim* s = nullptr;
  int rc = af::create(c, f, dem, h0, precision, device, &s);
  if (rc != AF_OK) return rc;
  *out = new af_sim{s};
  return AF_OK;
}

int af_sim_destroy(af_sim* h) {
  if (!h) return AF_EINVAL;
  cudaSetDevice(h->s->device);
  cudaStreamSynchronize(h->s->st);
  delete h->s;
  delete h;
  return AF_OK;
}

int af_sim_launch(af_sim* h, double t_stop, int64_t max_steps) {
  if (!h) return AF_EINVAL;
  return af::launch(*h->s, t_stop, max_steps);
}

int af_sim_sync(af_sim* h) {
  if (!h) return AF_EINVAL;
  AF_CUDA(cudaStreamSynchronize(h->s->st));
  AF_TRY(af::read_ctl(*h->s));
  return h->s->pinned_ctl->status ? AF_ESTATE : AF_OK;
}

int af_sim_run(af_sim* h, double t_stop, int64_t max_steps, int64_t* steps_done) {
  if (!h) return AF_EINVAL;
  Sim& s = *h->s;
  AF_TRY(af::read_ctl(s));
  long long before = s.pinned_ctl->step;
  AF_TRY(af::launch(s, t_stop, max_steps));
  AF_TRY(af::read_ctl(s));
  if (steps_done) *steps_done = s.pinned_ctl->step - before;
  return s.pinned_ctl->status ? AF_ESTATE : AF_OK;
}

int af_sim_status(af_sim* h, double* t, double* dt_last, double* hmax, int64_t* steps) {
  if (!h) return AF_EINVAL;
  Sim& s = *h->s;
  AF_TRY(af::read_ctl(s));
  if (t) *t = s.pinned_ctl->t;
  if (dt_last) *dt_last = s.pinned_ctl->dt_last;
  if (hmax) *hmax = s.pinned_ctl->hmax;
  if (steps) *steps = s.pinned_ctl->step;
  return AF_OK;
}

void* af_sim_stream(af_sim* h) { return h ? (void*)h->s->st : nullptr; }

int af_sim_get_state(af_sim* h, double* H, double* Qx, double* Qy) {
  if (!h) return AF_EINVAL;
  Sim& s = *h->s;
  AF_CUDA(cudaSetDevice(s.device));
  AF_TRY(af::read_ctl(s));
  const int par = s.pinned_ctl->parity;
  const int nx = s.c.nx, ny = s.c.ny;
  if (H) AF_TRY(af::get_field(s, s.H[par], H, ny, nx, nx));
  if (Qx) {
    AF_TRY(af::get_field(s, s.Qx[par], Qx, ny, nx + 1, nx + 1));
    for (int i = 0; i <= nx; i++) Qx[(size_t)ny * (nx + 1) + i] = 0.0;
  }
  if (Qy) {
    AF_TRY(af::get_field(s, s.Qy[par], Qy, ny + 1, nx, nx + 1));
    for (int j = 0; j <= ny; j++) Qy[(size_t)j * (nx + 1) + nx] = 0.0;
  }
  return AF_OK;
}

int af_sim_set_state(af_sim* h, const double* H, const double* Qx, const double* Qy, double t) {
  if (!h) return AF_EINVAL;
  Sim& s = *h->s;
  AF_CUDA(cudaSetDevice(s.device));
  AF_TRY(af::read_ctl(s));
  const int par = s.pinned_ctl->parity;
  const int nx = s.c.nx, ny = s.c.ny;
  if (H) AF_TRY(af::put_field(s, s.H[par], H, ny, nx, nx));
  if (Qx) AF_TRY(af::put_field(s, s.Qx[par], Qx, ny, nx + 1, nx + 1));
  if (Qy) AF_TRY(af::put_field(s, s.Qy[par], Qy, ny + 1, nx, nx + 1));
  af::SimCtl& c = *s.pinned_ctl;
  c.t = t;
  c.rain_rate = s.n_rain > 0 ? af::interp_series(s.rain_t.data(), s.rain_r.data(), s.n_rain, 0.0,
                                                 t, af::non_decreasing(s.rain_t.data(), s.n_rain))
                             : 0.0;
  c.next_mass = af::first_mass_after(t, s.c.mass_int);
  c.hmax_acc = af::ord_encode(-DBL_MAX);
  c.arrive = 0;
  c.done = 1;
  AF_TRY(af::write_ctl(s));
  AF_TRY(af::refresh_hmax(s, par));
  AF_CUDA(cudaStreamSynchronize(s.st));
  return AF_OK;
}

int af_sim_velocity(af_sim* h, double* Vx, double* Vy) {
  if (!h || !Vx || !Vy) return AF_EINVAL;
  Sim& s = *h->s;
  AF_CUDA(cudaSetDevice(s.device));
  AF_TRY(af::read_ctl(s));
  const int par = s.pinned_ctl->parity;
  const int nx = s.c.nx, ny = s.c.ny;
  const int rows_per = std::max(1, (int)((64LL << 20) / (16LL * nx)));
  af::DevBuf tmp;
  AF_TRY(af::alloc_field(tmp, (size_t)2 * rows_per * nx, 8));
  double* dvx = static_cast<double*>(tmp.p);
  double* dvy = dvx + (size_t)rows_per * nx;
  for (int j0 = 0; j0 < ny; j0 += rows_per) {
    int j1 = std::min(ny, j0 + rows_per);
    long long n = (long long)(j1 - j0) * nx;
    unsigned g = af::grid_for(n, 256, 8);
    if (s.prec == AF_PREC_F64)
      af::k_velocity_int<double><<<g, 256, 0, s.st>>>(
          s.buf<double>(s.H[par]), s.buf<double>(s.DEM), s.buf<double>(s.Qx[par]),
          s.buf<double>(s.Qy[par]), nx, j0, j1, s.P, s.c.dx, s.c.nodata, dvx, dvy);
    else
      af::k_velocity_int<float><<<g, 256, 0, s.st>>>(
          s.buf<float>(s.H[par]), s.buf<float>(s.DEM), s.buf<float>(s.Qx[par]),
          s.buf<float>(s.Qy[par]), nx, j0, j1, s.P, s.c.dx, s.c.nodata, dvx, dvy);
    AF_CUDA(cudaGetLastError());
    AF_CUDA(cudaMemcpyAsync(Vx + (size_t)j0 * nx, dvx, n * 8, cudaMemcpyDeviceToHost, s.st));
    AF_CUDA(cudaMemcpyAsync(Vy + (size_t)j0 * nx, dvy, n * 8, cudaMemcpyDeviceToHost, s.st));
  }
  AF_CUDA(cudaStreamSynchronize(s.st));
  return AF_OK;
}

int af_sim_volume(af_sim* h, double* vol, double* area) {
  if (!h || !vol || !area) return AF_EINVAL;
  Sim& s = *h->s;
  AF_CUDA(cudaSetDevice(s.device));
  AF_TRY(af::read_ctl(s));
  const int par = s.pinned_ctl->parity;
  const int nb = af::kSMs * 4;
  af::DevBuf part;
  AF_TRY(af::alloc_field(part, (size_t)nb * 3, 8));
  double dA = s.c.dx * s.c.dx;
  if (s.prec == AF_PREC_F64)
    af::k_volume_int<double><<<nb, 256, 0, s.st>>>(s.buf<double>(s.H[par]), s.c.nx, s.c.ny, s.P,
                                                   dA, static_cast<double*>(part.p));
  else
    af::k_volume_int<float><<<nb, 256, 0, s.st>>>(s.buf<float>(s.H[par]), s.c.nx, s.c.ny, s.P,
                                                  dA, static_cast<double*>(part.p));
  AF_CUDA(cudaGetLastError());
  std::vector<double> hp((size_t)nb * 3);
  AF_CUDA(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 8, cudaMemcpyDeviceToHost, s.st));
  AF_CUDA(cudaStreamSynchronize(s.st));
  double S = 0.0, C = 0.0, A = 0.0;
  for (int b = 0; b < nb; b++) {
    double x = hp[3 * b];
    double t = S + x;
    if (fabs(S) >= fabs(x)) C += (S - t) + x;
    else C += (x - t) + S;
    S = t;
    C += hp[3 * b + 1];
    A += hp[3 * b + 2];
  }
  *vol = S + C;
  *area = A;
  return AF_OK;
}

int af_sim_mass_series(af_sim* h, double* t, double* vol, double* area, int cap, int* n) {
  if (!h || !n || cap < 0) return AF_EINVAL;
  Sim& s = *h->s;
  AF_TRY(af::read_ctl(s));
  int cnt = std::min(s.pinned_ctl->mass_count, cap);
  std::vector<double> buf((size_t)std::max(cnt, 1) * 3);
  if (cnt > 0) {
    AF_CUDA(cudaMemcpyAsync(buf.data(), s.mass_series.p, (size_t)cnt * 24, cudaMemcpyDeviceToHost,
                            s.st));
    AF_CUDA(cudaStreamSynchronize(s.st));
  }
  for (int k = 0; k < cnt; k++) {
    if (t) t[k] = buf[3 * k];
    if (vol) vol[k] = buf[3 * k + 1];
    if (area) area[k] = buf[3 * k + 2];
  }
  *n = s.pinned_ctl->mass_count;
  return AF_OK;
}

}  // extern "C"

namespace af {

// The reference's main loop with its file outputs (src/main.cpp:196-388): the
// state at t = 0 as H_0000.asc, one save each time a step ends at or past the
// next save time, stage-point depths each time a step ends at or past the next
// stage time, and H_final.asc (+ Vx/Vy_final.asc) at the end.  The GPU keeps
// stepping while a save is copied out (copy stream) and written (writer
// thread): the snapshot kernel copies the state into a device buffer first.
static int run_output(Sim& s, double sim_time, const af_output_desc& o, int64_t* steps_out) {
  AF_CUDA(cudaSetDevice(s.device));
  if (!o.out_dir) return AF_EINVAL;
  if (::mkdir(o.out_dir, 0755) != 0 && errno != EEXIST) return AF_EIO;  // src/main.cpp:130
  const int nx = s.c.nx, ny = s.c.ny;
  const size_t cells = (size_t)nx * ny;
  const bool vel = o.voutput != 0;
  const int nf = vel ? 3 : 1;
  const int style = o.async_style ? kAscAsync : kAscSync;
  if (o.output_format < 0 || o.output_format > 2) return AF_EINVAL;
  // src/async_output.cpp:19, :144: the async writer writes NetCDF for formats
  // 1 and 2 and the periodic ASC grids for 0 and 2; the synchronous one ASC.
  const bool nc = o.async_style && o.output_format >= 1;
  const bool asc_saves = !o.async_style || o.output_format != 1;
  const std::string dir(o.out_dir);
  DevBuf dsnap, didx, dval;
  AF_TRY(alloc_field(dsnap, cells * nf, 8));
  std::unique_ptr<double, decltype(&cudaFreeHost)> hsnap(nullptr, &cudaFreeHost);
  std::unique_ptr<double, decltype(&cudaFreeHost)> hval(nullptr, &cudaFreeHost);
  {
    double* p = nullptr;
    AF_CUDA(cudaMallocHost((void**)&p, cells * nf * sizeof(double)));
    hsnap.reset(p);
  }
  struct Streams {
    cudaStream_t cst = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_copy = nullptr;
    ~Streams() {
      if (cst) cudaStreamSynchronize(cst);
      if (ev_snap) cudaEventDestroy(ev_snap);
      if (ev_copy) cudaEventDestroy(ev_copy);
      if (cst) cudaStreamDestroy(cst);
    }
  } R;
  AF_CUDA(cudaStreamCreateWithFlags(&R.cst, cudaStreamNonBlocking));
  AF_CUDA(cudaEventCreateWithFlags(&R.ev_snap, cudaEventDisableTiming));
  AF_CUDA(cudaEventCreateWithFlags(&R.ev_copy, cudaEventDisableTiming));
  AF_CUDA(cudaEventRecord(R.ev_copy, R.cst));
  const int nst = std::max(0, o.n_stage);
  FILE* stage_fp = nullptr;
  if (nst > 0) {
    std::vector<int> idx(o.stage_idx, o.stage_idx + nst);
    for (int& c : idx)
      if (c < 0 || (size_t)c >= cells) c = -1;
    AF_TRY(upload(didx, idx, s.st));
    AF_TRY(alloc_field(dval, nst, 8));
    double* p = nullptr;
    AF_CUDA(cudaMallocHost((void**)&p, nst * sizeof(double)));
    hval.reset(p);
    stage_fp = fopen((dir + "/stage.csv").c_str(), "w");  // src/main.cpp:100-108
    if (!stage_fp) return AF_EIO;
    fprintf(stage_fp, "Time(s)");
    for (int k = 0; k < nst; k++) {
      if (o.stage_names && o.stage_names[k]) fprintf(stage_fp, ",%s", o.stage_names[k]);
      else fprintf(stage_fp, ",Stage%d", k + 1);
    }
    fprintf(stage_fp, "\n");
  }
  std::unique_ptr<FILE, int (*)(FILE*)> stage_guard(stage_fp, [](FILE* f) {
    return f ? fclose(f) : 0;
  });
  std::unique_ptr<NcFile> ncf;  // declared before the writer, so it outlives its jobs
  if (nc) {
    ncf.reset(new NcFile);
    if (!ncf->open(dir + "/output.nc", nx, ny, vel, o.xll, o.yll, s.c.dx, s.c.nodata))
      return AF_EIO;
  }
  Writer writer;
  double* snap = static_cast<double*>(dsnap.p);

  // A save is two halves.  snapshot(): the state into the device buffer
  // (after the previous save's copy has left it), on the simulation stream,
  // before the next segment changes the state.  ship(): issued once the next
  // segment is queued, so the GPU keeps stepping meanwhile: the copy to pinned
  // host memory on the copy stream (after the writer has finished with it)
  // and the files on the writer thread.
  struct Pending {
    bool on = false;
    std::string tag;
    int style = 0;
    bool velocity = false;
    bool periodic = false;  // a save of the loop (ASC and/or NetCDF), not the final grids
    double t = 0.0;
  } pend;
  auto snapshot = [&](const std::string& tag, int st, bool velocity, bool periodic) -> int {
    AF_TRY(read_ctl(s));
    const int par = s.pinned_ctl->parity;
    AF_CUDA(cudaStreamWaitEvent(s.st, R.ev_copy, 0));
    const unsigned g = grid_for((long long)cells, 256, 8);
    double* vx = velocity ? snap + cells : nullptr;
    double* vy = velocity ? snap + 2 * cells : nullptr;
    if (s.prec == AF_PREC_F64)
      k_snapshot<double><<<g, 256, 0, s.st>>>(
          s.buf<double>(s.H[par]), s.buf<double>(s.DEM), s.buf<double>(s.Qx[par]),
          s.buf<double>(s.Qy[par]), nx, ny, s.P, s.c.dx, s.c.nodata, snap, vx, vy);
    else
      k_snapshot<float><<<g, 256, 0, s.st>>>(
          s.buf<float>(s.H[par]), s.buf<float>(s.DEM), s.buf<float>(s.Qx[par]),
          s.buf<float>(s.Qy[par]), nx, ny, s.P, s.c.dx, s.c.nodata, snap, vx, vy);
    AF_CUDA(cudaGetLastError());
    AF_CUDA(cudaEventRecord(R.ev_snap, s.st));
    pend.on = true;
    pend.tag = tag;
    pend.style = st;
    pend.velocity = velocity;
    pend.periodic = periodic;
    pend.t = s.pinned_ctl->t;
    return AF_OK;
  };
  auto ship = [&]() -> int {
    if (!pend.on) return AF_OK;
    pend.on = false;
    writer.drain();  // the pinned copy is free again
    const bool velocity = pend.velocity;
    const size_t nb = cells * (velocity ? 3 : 1) * sizeof(double);
    AF_CUDA(cudaStreamWaitEvent(R.cst, R.ev_snap, 0));
    AF_CUDA(cudaMemcpyAsync(hsnap.get(), snap, nb, cudaMemcpyDeviceToHost, R.cst));
    AF_CUDA(cudaEventRecord(R.ev_copy, R.cst));
    const double* h = hsnap.get();
    const double xll = o.xll, yll = o.yll, cs = s.c.dx, nd = s.c.nodata;
    const std::string tag = pend.tag;
    const int st = pend.style;
    const bool asc = !pend.periodic || asc_saves;
    NcFile* ncp = pend.periodic ? ncf.get() : nullptr;
    const double ts = pend.t;
    cudaEvent_t ev = R.ev_copy;
    writer.post([&writer, h, cells, dir, tag, st, velocity, nx, ny, xll, yll, cs, nd, ev, asc,
                 ncp, ts] {
      if (cudaEventSynchronize(ev) != cudaSuccess) {
        writer.fail();
        return;
      }
      const char* names[3] = {"H", "Vx", "Vy"};
      for (int f = 0; asc && f < (velocity ? 3 : 1); f++) {
        const std::string path = dir + "/" + names[f] + "_" + tag + ".asc";
        if (!write_asc(path.c_str(), h + f * cells, nx, ny, xll, yll, cs, nd, st, 0))
          writer.fail();
      }
      if (ncp && !ncp->append(ts, h, velocity ? h + cells : nullptr,
                              velocity ? h + 2 * cells : nullptr))
        writer.fail();
    });
    return AF_OK;
  };
  auto tag_of = [](int n) {
    char b[16];
    snprintf(b, sizeof b, "%04d", n);
    return std::string(b);
  };

  AF_TRY(read_ctl(s));
  const long long step0 = s.pinned_ctl->step;
  double t = s.pinned_ctl->t;
  int save_num = 0;
  AF_TRY(snapshot(tag_of(save_num++), style, vel && style == kAscAsync, true));  // src/main.cpp:206-225
  const double inf = 1e300;
  double next_save = o.save_int > 0.0 ? o.save_int : inf;  // src/main.cpp:199-201
  double next_stage = (nst > 0 && o.stage_int > 0.0) ? o.stage_int : inf;
  while (t < sim_time) {  // src/main.cpp:227
    const double stop = std::min(sim_time, std::min(next_save, next_stage));
    // At least one step: a save or stage time already passed is taken after
    // the next step, one per step, as the reference's loop does.
    if (t < stop) AF_TRY(launch(s, stop, 0x3FFFFFFFFFFFFFFFLL));
    else AF_TRY(launch(s, sim_time, 1));
    AF_TRY(ship());  // the previous save leaves while this segment runs
    AF_CUDA(cudaStreamSynchronize(s.st));
    AF_TRY(read_ctl(s));
    if (s.pinned_ctl->status) return AF_ESTATE;
    t = s.pinned_ctl->t;
    if (nst > 0 && t >= next_stage) {  // src/main.cpp:306-322
      const int par = s.pinned_ctl->parity;
      if (s.prec == AF_PREC_F64)
        k_gather<double><<<(nst + 127) / 128, 128, 0, s.st>>>(
            s.buf<double>(s.H[par]), nx, s.P, (const int*)didx.p, nst, (double*)dval.p);
      else
        k_gather<float><<<(nst + 127) / 128, 128, 0, s.st>>>(
            s.buf<float>(s.H[par]), nx, s.P, (const int*)didx.p, nst, (double*)dval.p);
      AF_CUDA(cudaMemcpyAsync(hval.get(), dval.p, nst * sizeof(double), cudaMemcpyDeviceToHost,
                              s.st));
      AF_CUDA(cudaStreamSynchronize(s.st));
      fprintf(stage_fp, "%.1f", t);
      for (int k = 0; k < nst; k++) {
        const int c = o.stage_idx[k];
        if (c >= 0 && (size_t)c < cells) fprintf(stage_fp, ",%.4f", hval.get()[k]);
        else fprintf(stage_fp, ",NaN");
      }
      fprintf(stage_fp, "\n");
      fflush(stage_fp);
      next_stage += o.stage_int;
    }
    if (t >= next_save) {  // src/main.cpp:325-363
      AF_TRY(snapshot(tag_of(save_num++), style, vel && style == kAscAsync, true));
      next_save += o.save_int;
    }
  }
  AF_TRY(ship());
  // Final state (src/main.cpp:376-388): always the synchronous writer's format.
  AF_TRY(snapshot("final", kAscSync, vel, false));
  AF_TRY(ship());
  writer.drain();
  if (steps_out) *steps_out = s.pinned_ctl->step - step0;
  return writer.errors() ? AF_EIO : AF_OK;
}

// Checkpoint file: "AFCKPT02", int32 precision, nx, ny, mass count, uint32
// sizeof(SimCtl), uint32 0, uint64 hash of the case parameters and forcing,
// uint64 hash of the stored DEM, the control block (SimCtl, native layout),
// the mass series (3 doubles per entry), then H (ny x nx), Qx (ny x (nx+1))
// and Qy ((ny+1) x nx) in the state precision, dense.  Native byte order: a
// checkpoint is read back on the same kind of host it was written on.  A
// restore into another case (grid, parameters, forcing or DEM), precision or
// build whose control block differs is refused with AF_EINVAL.
static const char kCkptMagic[8] = {'A', 'F', 'C', 'K', 'P', 'T', '0', '2'};

// (The accumulator is the first word of the step's partials buffer, which
// holds nothing between launches; stream order puts this after any step.)
static int dem_hash(Sim& s, uint64_t* out) {
  DevBuf& acc = s.partials;
  AF_CUDA(cudaMemsetAsync(acc.p, 0, 8, s.st));
  const long long n = (long long)s.c.nx * s.c.ny;
  const unsigned grid = grid_for(n, 256, 4);
  unsigned long long* a = static_cast<unsigned long long*>(acc.p);
  if (s.prec == AF_PREC_F64)
    k_dem_hash<double><<<grid, 256, 0, s.st>>>(s.buf<double>(s.DEM), s.c.nx, s.c.ny, s.P, a);
  else
    k_dem_hash<float><<<grid, 256, 0, s.st>>>(s.buf<float>(s.DEM), s.c.nx, s.c.ny, s.P, a);
  AF_CUDA(cudaGetLastError());
  unsigned long long h = 0;
  AF_CUDA(cudaMemcpyAsync(&h, acc.p, 8, cudaMemcpyDeviceToHost, s.st));
  AF_CUDA(cudaStreamSynchronize(s.st));
  *out = h;
  return AF_OK;
}

static int field_io(Sim& s, DevBuf& b, std::vector<char>& host, int rows, int width, bool put) {
  char* dev = static_cast<char*>(b.p) + (size_t)kGuard * s.esize;
  const size_t w = (size_t)width * s.esize;
  if (put)
    AF_CUDA(copy2d_h2d(dev, (size_t)s.P * s.esize, host.data(), w, w, rows, s.st));
  else
    AF_CUDA(copy2d_d2h(host.data(), w, dev, (size_t)s.P * s.esize, w, rows, s.st));
  AF_CUDA(cudaStreamSynchronize(s.st));
  return AF_OK;
}

static int checkpoint(Sim& s, const char* path) {
  AF_CUDA(cudaSetDevice(s.device));
  AF_TRY(read_ctl(s));
  const SimCtl ctl = *s.pinned_ctl;
  const int par = ctl.parity, nx = s.c.nx, ny = s.c.ny;
  const int nm = std::min(ctl.mass_count, ctl.mass_cap);
  std::vector<double> mass((size_t)nm * 3);
  if (nm > 0) {
    AF_CUDA(cudaMemcpyAsync(mass.data(), s.mass_series.p, mass.size() * 8, cudaMemcpyDeviceToHost,
                            s.st));
    AF_CUDA(cudaStreamSynchronize(s.st));
  }
  FILE* f = fopen(path, "wb");
  if (!f) return AF_EIO;
  std::unique_ptr<FILE, int (*)(FILE*)> guard(f, fclose);
  const int32_t hdr[4] = {s.prec, nx, ny, nm};
  const uint32_t sizes[2] = {(uint32_t)sizeof(SimCtl), 0u};
  uint64_t ids[2] = {s.case_hash, 0};
  AF_TRY(dem_hash(s, &ids[1]));
  bool ok = fwrite(kCkptMagic, 1, 8, f) == 8 && fwrite(hdr, sizeof hdr, 1, f) == 1 &&
            fwrite(sizes, sizeof sizes, 1, f) == 1 && fwrite(ids, sizeof ids, 1, f) == 1 &&
            fwrite(&ctl, sizeof ctl, 1, f) == 1 &&
            (nm == 0 || fwrite(mass.data(), 8, mass.size(), f) == mass.size());
  const int shape[3][2] = {{ny, nx}, {ny, nx + 1}, {ny + 1, nx}};
  DevBuf* fields[3] = {&s.H[par], &s.Qx[par], &s.Qy[par]};
  for (int k = 0; k < 3 && ok; k++) {
    std::vector<char> host((size_t)shape[k][0] * shape[k][1] * s.esize);
    AF_TRY(field_io(s, *fields[k], host, shape[k][0], shape[k][1], false));
    ok = fwrite(host.data(), 1, host.size(), f) == host.size();
  }
  guard.reset();
  return ok ? AF_OK : AF_EIO;
}

static int restore(Sim& s, const char* path) {
  AF_CUDA(cudaSetDevice(s.device));
  FILE* f = fopen(path, "rb");
  if (!f) return AF_EIO;
  std::unique_ptr<FILE, int (*)(FILE*)> guard(f, fclose);
  char magic[8];
  int32_t hdr[4];
  uint32_t sizes[2];
  uint64_t ids[2];
  SimCtl ctl;
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kCkptMagic, 8) != 0 ||
      fread(hdr, sizeof hdr, 1, f) != 1 || fread(sizes, sizeof sizes, 1, f) != 1 ||
      fread(ids, sizeof ids, 1, f) != 1)
    return AF_EIO;
  const int nx = s.c.nx, ny = s.c.ny;
  if (sizes[0] != (uint32_t)sizeof(SimCtl) || hdr[0] != s.prec || hdr[1] != nx ||
      hdr[2] != ny || hdr[3] < 0 || hdr[3] > kMassCap || ids[0] != s.case_hash)
    return AF_EINVAL;  // another case, precision or control-block layout
  uint64_t dem_id = 0;
  AF_TRY(dem_hash(s, &dem_id));
  if (ids[1] != dem_id) return AF_EINVAL;  // another DEM
  if (fread(&ctl, sizeof ctl, 1, f) != 1) return AF_EIO;
  if (ctl.parity < 0 || ctl.parity > 1) return AF_EINVAL;
  std::vector<double> mass((size_t)hdr[3] * 3);
  if (!mass.empty() && fread(mass.data(), 8, mass.size(), f) != mass.size()) return AF_EIO;
  const int par = ctl.parity;
  const int shape[3][2] = {{ny, nx}, {ny, nx + 1}, {ny + 1, nx}};
  DevBuf* fields[3] = {&s.H[par], &s.Qx[par], &s.Qy[par]};
  std::vector<std::vector<char>> host(3);
  for (int k = 0; k < 3; k++) {
    host[k].resize((size_t)shape[k][0] * shape[k][1] * s.esize);
    if (fread(host[k].data(), 1, host[k].size(), f) != host[k].size()) return AF_EIO;
  }
  for (int k = 0; k < 3; k++) AF_TRY(field_io(s, *fields[k], host[k], shape[k][0], shape[k][1], true));
  if (!mass.empty()) {
    AF_CUDA(cudaMemcpyAsync(s.mass_series.p, mass.data(), mass.size() * 8, cudaMemcpyHostToDevice,
                            s.st));
    AF_CUDA(cudaStreamSynchronize(s.st));
  }
  ctl.mass_count = hdr[3];
  ctl.mass_cap = kMassCap;
  ctl.hmax_acc = ord_encode(-DBL_MAX);
  ctl.arrive = 0;
  ctl.done = 1;
  ctl.status = 0;
  *s.pinned_ctl = ctl;
  return write_ctl(s);
}

}  // namespace af

extern "C" {

int af_sim_checkpoint(af_sim* h, const char* path) {
  if (!h || !path) return AF_EINVAL;
  return af::checkpoint(*h->s, path);
}

int af_sim_restore(af_sim* h, const char* path) {
  if (!h || !path) return AF_EINVAL;
  return af::restore(*h->s, path);
}

int af_sim_run_output(af_sim* h, double sim_time, const af_output_desc* o, int64_t* steps) {
  if (!h || !o) return AF_EINVAL;
  return af::run_output(*h->s, sim_time, *o, steps);
}

}  // extern "C"
