// af_batch.cu -- the batch engine: many independent grids ("scenarios") of
// uneven sizes, each with its own parameters, forcing, adaptive dt and stop
// time, stepped together by one persistent kernel inside one CUDA graph.
//
// Memory: one device arena taken at creation (af_batch_create's arena_bytes)
// holds every scenario's padded fields (af_simcore.cuh layout) and tables;
// the host-side planner (af_arena.h) places them, so admitting and retiring
// scenarios never allocates or frees device memory while others run.  A
// scenario is admitted only if its footprint fits (AF_ENOMEM otherwise, with
// nothing changed), which is the admission-by-HBM-footprint rule of the
// serving loop.
//
// Control: per slot a SimCtl (time, dt inputs, parity, counters) in one
// device array; the batch's member list and active list in a BatchTab; the
// loop state in a BatchCtl.  A launch runs batch steps (every active
// scenario advances one step of its own dt) until nothing is active, a step
// limit is reached, a scenario finishes (stop_on_done), or the host raises the
// attention flag (host memory mapped into the device).
//
// Concurrency rules (one host thread drives a batch):
//   * af_batch_add may run while a launch is in flight: its uploads go on a
//     separate copy stream into arena space and a slot no running launch
//     reads; the scenario joins at the next launch.
//   * af_batch_remove while a launch is in flight defers the release of the
//     slot and its arena space to the next af_batch_sync.
//   * af_batch_get_state may run while a launch is in flight for a scenario
//     that had finished at the last sync (it is no longer stepped).
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "af_arena.h"
#include "af_simcore.cuh"
#include "af_xfer.h"

namespace af {

constexpr int kClasses = 32;  // size class = floor(log2(nx*ny))
constexpr int kBatchMassCap = 1 << 16;

static int size_class(long long cells) {
  int c = 0;
  while (c + 1 < kClasses && (1LL << (c + 1)) <= cells) c++;
  return c;
}

// Default strip height per size class, used until a tuned table is set.
static int default_rows(int cls) {
  if (cls < 16) return 4;
  if (cls < 20) return 8;
  if (cls < 24) return 16;
  return 32;
}

static size_t align_up(size_t x) { return (x + Arena::kAlign - 1) / Arena::kAlign * Arena::kAlign; }

// Byte offsets of one scenario's arrays inside its arena block.
struct Layout {
  int nx = 0, ny = 0, P = 0, R = 0, nsx = 0, nsy = 0;
  size_t H[2], Qx[2], Qy[2], DEM;
  size_t src_type, src_value, src_off, src_times, src_vals, src_sorted;
  size_t bc_type, bc_value, bc_off, bc_times, bc_vals, bc_sorted;
  size_t rain_times, rain_rates, spec_off, spec, partials, mass;
  int mass_cap = 0;
  size_t total = 0;
};

static int series_len(const int* off, const int* type, int n, int want_type) {
  int s = 0;
  for (int k = 0; k < n; k++)
    if (type[k] == want_type) s += off[k + 1] - off[k];
  return s;
}

static Layout make_layout(const af_case_desc* c, const af_forcing_desc* f, double t_stop, int R,
                          int esize) {
  Layout L;
  const int N = 16 / esize;
  L.nx = c->nx;
  L.ny = c->ny;
  L.P = row_pitch(c->nx, N);
  L.R = R;
  L.nsx = strips_x(c->nx, N);
  L.nsy = (c->ny + R - 1) / R;
  size_t at = 0;
  auto put = [&](size_t bytes) {
    const size_t o = at;
    at += align_up(std::max<size_t>(bytes, 1));
    return o;
  };
  const size_t cb = cell_elems(L.ny, L.P) * esize, qb = qy_elems(L.ny, L.P) * esize;
  for (int b = 0; b < 2; b++) {
    L.H[b] = put(cb);
    L.Qx[b] = put(cb);
    L.Qy[b] = put(qb);
  }
  L.DEM = put(cb);
  const int nf = f->n_flow, no = f->n_other;
  const int sl = series_len(f->flow_off, f->flow_type, nf, AF_BC_QVAR);
  const int bl = series_len(f->other_off, f->other_type, no, AF_BC_HVAR);
  L.src_type = put(sizeof(int) * nf);
  L.src_value = put(sizeof(double) * nf);
  L.src_off = put(sizeof(int) * (nf + 1));
  L.src_times = put(sizeof(double) * sl);
  L.src_vals = put(sizeof(double) * sl);
  L.src_sorted = put(nf);
  L.bc_type = put(sizeof(int) * no);
  L.bc_value = put(sizeof(double) * no);
  L.bc_off = put(sizeof(int) * (no + 1));
  L.bc_times = put(sizeof(double) * bl);
  L.bc_vals = put(sizeof(double) * bl);
  L.bc_sorted = put(no);
  L.rain_times = put(sizeof(double) * f->n_rain);
  L.rain_rates = put(sizeof(double) * f->n_rain);
  // Per-strip arrays are sized for one-row strips, so the strip height can
  // change between launches without moving anything.
  const size_t nstrips = (size_t)L.nsx * L.ny;
  L.spec_off = put(sizeof(int) * (nstrips + 1));
  L.spec = put(sizeof(SpecCell) * (size_t)(nf + no));  // at most one per source or BC
  L.partials = put(sizeof(double) * 3 * nstrips);
  long long cap = 2;
  if (c->mass_int > 0.0 && t_stop > 0.0 && t_stop < 1e300)
    cap = (long long)std::ceil(t_stop / c->mass_int) + 2;
  L.mass_cap = (int)std::min<long long>(std::max<long long>(cap, 2), kBatchMassCap);
  L.mass = put(sizeof(double) * 3 * L.mass_cap);
  L.total = at;
  return L;
}

struct Slot {
  int state = 0;  // 0 free, 1 member, 2 released at the next sync
  uint64_t off = 0;
  Layout L;
  af_case_desc c{};
  double t_stop = 0.0;
  int cls = 0;                  // size class
  std::vector<SpecCell> spec;   // special cells in (column strip, row, col) order
  StepParams p{};               // the device copy's host image
};

struct Batch {
  int device = 0, prec = AF_PREC_F32, esize = 4, N = 4, variant = 0, WY = 1;
  cudaStream_t st = nullptr, cst = nullptr;
  char* arena = nullptr;
  Arena plan;
  double* stage = nullptr;  // kStageBytes of FP64 staging for FP32 field transfers
  BatchScen* d_scen = nullptr;
  SimCtl* d_ctl = nullptr;
  BatchTab* d_tab = nullptr;
  BatchCtl* d_bctl = nullptr;
  SimCtl* h_ctl = nullptr;    // pinned mirror of d_ctl, refreshed by sync
  BatchTab* h_tab = nullptr;  // pinned staging of the member list
  BatchCtl* h_bctl = nullptr;
  int* h_attn = nullptr;      // mapped pinned attention flag
  int* d_attn = nullptr;
  unsigned long long* d_trace = nullptr;  // per-step trace records (af_batch_set_trace)
  BatchParams bp{};
  dim3 grid, block;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t begin_node = nullptr;
  cudaGraphConditionalHandle cond = 0;
  bool use_cond = false;
  bool in_flight = false;
  bool members_dirty = true;
  int balance = 4;  // strips per warp the load-adaptive strip height aims at (0: off)
  int hi_slot = 0;  // one past the highest slot ever used
  int rows[kClasses];
  std::vector<Slot> slots;

  ~Batch() {
    if (device >= 0) cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    if (cst) cudaStreamSynchronize(cst);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (arena) cudaFree(arena);
    if (stage) cudaFree(stage);
    if (d_scen) cudaFree(d_scen);
    if (d_ctl) cudaFree(d_ctl);
    if (d_tab) cudaFree(d_tab);
    if (d_bctl) cudaFree(d_bctl);
    if (d_trace) cudaFree(d_trace);
    if (h_ctl) cudaFreeHost(h_ctl);
    if (h_tab) cudaFreeHost(h_tab);
    if (h_bctl) cudaFreeHost(h_bctl);
    if (h_attn) cudaFreeHost(h_attn);
    if (st) cudaStreamDestroy(st);
    if (cst) cudaStreamDestroy(cst);
  }

  const void* kernel() const {
    return prec == AF_PREC_F64 ? batch_kernel_f64(variant) : batch_kernel_f32(variant);
  }
  const void* begin_kernel() const {
    return prec == AF_PREC_F64 ? batch_begin_f64() : batch_begin_f32();
  }
  const void* fold_kernel() const {
    return prec == AF_PREC_F64 ? batch_fold_f64() : batch_fold_f32();
  }
};

static int alloc_dev(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cuda_fail(e);
    return AF_ENOMEM;
  }
  return AF_OK;
}

static int build_graph(Batch& b) {
  b.bp.scen = b.d_scen;
  b.bp.tab = b.d_tab;
  b.bp.bctl = b.d_bctl;
  b.bp.attention = b.d_attn;
  const char* direct = getenv("AF_SIM_DIRECT_LAUNCH");
  if (direct && direct[0] && direct[0] != '0') return AF_OK;
  AF_CUDA(cudaGraphCreate(&b.graph, 0));
  b.use_cond = cudaGraphConditionalHandleCreate(&b.cond, b.graph, 0, 0) == cudaSuccess;
  if (!b.use_cond) {
    cudaGetLastError();
    cudaGraphDestroy(b.graph);
    b.graph = nullptr;
    return AF_OK;  // host-driven launches
  }
  b.bp.cond = b.cond;
  b.bp.use_cond = 1;
  long long max_steps = 0;
  int stop_on_done = 0;
  void* bargs[] = {&b.bp, &max_steps, &stop_on_done};
  cudaKernelNodeParams kb{};
  kb.func = const_cast<void*>(b.begin_kernel());
  kb.gridDim = dim3(1);
  kb.blockDim = dim3(kFoldThreads);
  kb.kernelParams = bargs;
  AF_CUDA(cudaGraphAddKernelNode(&b.begin_node, b.graph, nullptr, 0, &kb));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = b.cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  AF_CUDA(cudaGraphAddNode(&cnode, b.graph, &b.begin_node, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // Body: kStepsPerIteration batch steps, each the strips of every active
  // scenario, then the fold.
  void* sargs[] = {&b.bp};
  cudaKernelNodeParams ks{};
  ks.func = const_cast<void*>(b.kernel());
  ks.gridDim = b.grid;
  ks.blockDim = b.block;
  ks.kernelParams = sargs;
  cudaKernelNodeParams kf{};
  kf.func = const_cast<void*>(b.fold_kernel());
  kf.gridDim = dim3(1);
  kf.blockDim = dim3(kFoldThreads);
  kf.kernelParams = sargs;
  cudaGraphNode_t prev = nullptr;
  for (int k = 0; k < kStepsPerIteration; k++) {
    cudaGraphNode_t snode, fnode;
    AF_CUDA(cudaGraphAddKernelNode(&snode, body, prev ? &prev : nullptr, prev ? 1 : 0, &ks));
    AF_CUDA(cudaGraphAddKernelNode(&fnode, body, &snode, 1, &kf));
    prev = fnode;
  }
  AF_CUDA(cudaGraphInstantiate(&b.exec, b.graph, 0));
  return AF_OK;
}

static int create(int precision, int device, uint64_t arena_bytes, int variant, Batch** out) {
  if (!out) return AF_EINVAL;
  if (precision != AF_PREC_F64 && precision != AF_PREC_F32) return AF_EINVAL;
  if (arena_bytes < Arena::kAlign) return AF_EINVAL;
  std::unique_ptr<Batch> b(new (std::nothrow) Batch());
  if (!b) return AF_ENOMEM;
  b->device = device;
  b->prec = precision;
  b->esize = precision == AF_PREC_F64 ? 8 : 4;
  b->N = 16 / b->esize;
  if (variant < 0) {
    // Default: 1 warp per block with 16 resident blocks per SM in FP32 (128
    // registers, no spills: the fastest shape on every measured mix), 12 in
    // FP64 (whose 16-block shape spills).
    variant = precision == AF_PREC_F32 ? 0 : 1;
    if (const char* v = getenv("AF_BATCH_VARIANT")) variant = atoi(v);
  }
  if (variant < 0 || variant >= kStepVariants) return AF_EINVAL;
  b->variant = variant;
  b->WY = kStepVariant[variant].wy;
  for (int k = 0; k < kClasses; k++) b->rows[k] = default_rows(k);
  b->slots.resize(kMaxSlots);
  AF_CUDA(cudaSetDevice(device));
  AF_CUDA(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
  AF_CUDA(cudaStreamCreateWithFlags(&b->cst, cudaStreamNonBlocking));
  AF_TRY(alloc_dev((void**)&b->arena, arena_bytes));
  AF_TRY(alloc_dev((void**)&b->stage, kStageBytes));
  b->plan.reset(arena_bytes);
  AF_TRY(alloc_dev((void**)&b->d_scen, sizeof(BatchScen) * kMaxSlots));
  AF_TRY(alloc_dev((void**)&b->d_ctl, sizeof(SimCtl) * kMaxSlots));
  AF_TRY(alloc_dev((void**)&b->d_tab, sizeof(BatchTab)));
  AF_TRY(alloc_dev((void**)&b->d_bctl, sizeof(BatchCtl)));
  AF_CUDA(cudaMemsetAsync(b->d_scen, 0, sizeof(BatchScen) * kMaxSlots, b->st));
  AF_CUDA(cudaMemsetAsync(b->d_ctl, 0, sizeof(SimCtl) * kMaxSlots, b->st));
  AF_CUDA(cudaMemsetAsync(b->d_tab, 0, sizeof(BatchTab), b->st));
  AF_CUDA(cudaMemsetAsync(b->d_bctl, 0, sizeof(BatchCtl), b->st));
  AF_CUDA(cudaMallocHost((void**)&b->h_ctl, sizeof(SimCtl) * kMaxSlots));
  AF_CUDA(cudaMallocHost((void**)&b->h_tab, sizeof(BatchTab)));
  AF_CUDA(cudaMallocHost((void**)&b->h_bctl, sizeof(BatchCtl)));
  AF_CUDA(cudaHostAlloc((void**)&b->h_attn, sizeof(int), cudaHostAllocMapped));
  AF_CUDA(cudaHostGetDevicePointer((void**)&b->d_attn, b->h_attn, 0));
  memset(b->h_ctl, 0, sizeof(SimCtl) * kMaxSlots);
  memset(b->h_tab, 0, sizeof(BatchTab));
  memset(b->h_bctl, 0, sizeof(BatchCtl));
  *b->h_attn = 0;
  // Persistent grid: every block resident at once.
  int per_sm = 0, sms = kSMs;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->kernel(), 32 * b->WY, 0) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  b->grid = dim3((unsigned)(sms * per_sm));
  b->block = dim3(32 * b->WY);
  AF_TRY(build_graph(*b));
  AF_CUDA(cudaStreamSynchronize(b->st));
  *out = b.release();
  return AF_OK;
}

// Uploads `bytes` from a host vector into the arena (copy stream).
template <typename V>
static int put_vec(Batch& b, char* base, size_t off, const std::vector<V>& v) {
  if (v.empty()) return AF_OK;
  AF_CUDA(cudaMemcpyAsync(base + off, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice,
                          b.cst));
  return AF_OK;
}

// Caller FP64 rows -> a padded field in the arena (`dst` = the field's
// allocation, front guard included), on the copy stream: FP64 in one 2-D copy,
// FP32 through the staging buffer and a conversion kernel.
template <typename T>
static int put_padded(Batch& b, char* dst, const double* src, int rows, int width, int P) {
  T* d = reinterpret_cast<T*>(dst) + kGuard;
  if (sizeof(T) == 8) {
    AF_CUDA(copy2d_h2d(d, (size_t)P * 8, src, (size_t)width * 8, (size_t)width * 8, rows, b.cst));
  } else {
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(rows, kStageBytes / (8 * (size_t)width)));
    for (int j = 0; j < rows; j += chunk) {
      const int n = std::min(chunk, rows - j);
      AF_CUDA(copy2d_h2d(b.stage, (size_t)width * 8, src + (size_t)j * width, (size_t)width * 8,
                         (size_t)width * 8, n, b.cst));
      k_pad_from_f64<<<grid_for((long long)n * width, 256, 8), 256, 0, b.cst>>>(
          b.stage, n, width, reinterpret_cast<float*>(d) + (size_t)j * P, P);
      AF_CUDA(cudaGetLastError());
    }
  }
  AF_CUDA(cudaStreamSynchronize(b.cst));
  return AF_OK;
}

static int add(Batch& b, const af_case_desc* c, const af_forcing_desc* f, const double* dem,
               const double* h0, double t_stop, int* slot_out) {
  if (!c || !f || !dem || !slot_out) return AF_EINVAL;
  AF_TRY(check_case(c, f));
  if (!(t_stop == t_stop)) return AF_EINVAL;
  int slot = -1;
  for (int k = 0; k < kMaxSlots; k++)
    if (b.slots[k].state == 0) {
      slot = k;
      break;
    }
  if (slot < 0) return AF_ENOMEM;
  const int R = b.rows[size_class((long long)c->nx * c->ny)];
  const Layout L = make_layout(c, f, t_stop, R, b.esize);
  uint64_t off = 0;
  if (!b.plan.alloc(L.total, &off)) return AF_ENOMEM;
  AF_CUDA(cudaSetDevice(b.device));
  auto fail = [&](int rc) {
    b.plan.release(off);
    return rc;
  };
  HostTables tb;
  build_tables(c, f, 30 * b.N, R, L.nsx, L.nsy, tb);
  char* base = b.arena + off;
  int rc = AF_OK;
  if (cudaMemsetAsync(base, 0, L.total, b.cst) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError()));
  if (b.prec == AF_PREC_F64) {
    rc = put_padded<double>(b, base + L.DEM, dem, L.ny, L.nx, L.P);
    if (rc == AF_OK && h0) rc = put_padded<double>(b, base + L.H[0], h0, L.ny, L.nx, L.P);
  } else {
    rc = put_padded<float>(b, base + L.DEM, dem, L.ny, L.nx, L.P);
    if (rc == AF_OK && h0) rc = put_padded<float>(b, base + L.H[0], h0, L.ny, L.nx, L.P);
  }
  if (rc != AF_OK) return fail(rc);
  const int puts[] = {
      put_vec(b, base, L.src_type, tb.src_type),   put_vec(b, base, L.src_value, tb.src_value),
      put_vec(b, base, L.src_off, tb.src_off),     put_vec(b, base, L.src_times, tb.src_times),
      put_vec(b, base, L.src_vals, tb.src_vals),   put_vec(b, base, L.src_sorted, tb.src_sorted),
      put_vec(b, base, L.bc_type, tb.bc_type),     put_vec(b, base, L.bc_value, tb.bc_value),
      put_vec(b, base, L.bc_off, tb.bc_off),       put_vec(b, base, L.bc_times, tb.bc_times),
      put_vec(b, base, L.bc_vals, tb.bc_vals),     put_vec(b, base, L.bc_sorted, tb.bc_sorted),
      put_vec(b, base, L.rain_times, tb.rain_times), put_vec(b, base, L.rain_rates, tb.rain_rates),
      put_vec(b, base, L.spec_off, tb.spec_off),   put_vec(b, base, L.spec, tb.spec)};
  for (int r : puts)
    if (r != AF_OK) return fail(r);

  StepParams p{};
  const size_t g = (size_t)kGuard * b.esize;
  for (int k = 0; k < 2; k++) {
    p.H[k] = base + L.H[k] + g;
    p.Qx[k] = base + L.Qx[k] + g;
    p.Qy[k] = base + L.Qy[k] + g;
  }
  p.DEM = base + L.DEM + g;
  p.nx = L.nx;
  p.ny = L.ny;
  p.P = L.P;
  p.nsx = L.nsx;
  p.nsy = L.nsy;
  p.R = L.R;
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
  {
    // Whether the stored DEM has a nodata cell (the first word of the
    // scenario's strip partials, unused until it is stepped, as the flag).
    int* flag = (int*)(base + L.partials);
    const unsigned gn = grid_for((long long)L.nx * L.ny, 256, 8);
    cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), b.cst);
    if (e == cudaSuccess) {
      if (b.prec == AF_PREC_F64)
        k_any_nodata<double><<<gn, 256, 0, b.cst>>>((const double*)p.DEM, L.nx, L.ny, L.P,
                                                    c->nodata, flag);
      else
        k_any_nodata<float><<<gn, 256, 0, b.cst>>>((const float*)p.DEM, L.nx, L.ny, L.P,
                                                   c->nodata, flag);
      e = cudaGetLastError();
    }
    int hflag = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost,
                                              b.cst);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b.cst);
    if (e != cudaSuccess) return fail(cuda_fail(e));
    p.has_nodata = hflag;
  }
  p.src_type = (const int*)(base + L.src_type);
  p.src_value = (const double*)(base + L.src_value);
  p.src_off = (const int*)(base + L.src_off);
  p.src_times = (const double*)(base + L.src_times);
  p.src_vals = (const double*)(base + L.src_vals);
  p.src_sorted = (const unsigned char*)(base + L.src_sorted);
  p.bc_type = (const int*)(base + L.bc_type);
  p.bc_value = (const double*)(base + L.bc_value);
  p.bc_off = (const int*)(base + L.bc_off);
  p.bc_times = (const double*)(base + L.bc_times);
  p.bc_vals = (const double*)(base + L.bc_vals);
  p.bc_sorted = (const unsigned char*)(base + L.bc_sorted);
  p.rain_times = (const double*)(base + L.rain_times);
  p.rain_rates = (const double*)(base + L.rain_rates);
  p.n_rain = f->n_rain;
  p.rain_sorted = tb.rain_sorted;
  p.spec_off = (const int*)(base + L.spec_off);
  p.spec = (const SpecCell*)(base + L.spec);
  p.ctl = b.d_ctl + slot;
  p.partials = (double*)(base + L.partials);
  p.mass_series = (double*)(base + L.mass);
  p.use_cond = 0;

  SimCtl h{};
  h.t = 0.0;
  h.hmax = -DBL_MAX;
  h.rain_rate = f->n_rain > 0 ? interp_series(tb.rain_times.data(), tb.rain_rates.data(),
                                              f->n_rain, 0.0, 0.0, tb.rain_sorted != 0)
                              : 0.0;
  h.t_stop = t_stop;
  h.next_mass = first_mass_after(0.0, c->mass_int);
  h.step_stop = 0x3FFFFFFFFFFFFFFFLL;
  h.hmax_acc = ord_encode(-DBL_MAX);
  h.mass_cap = L.mass_cap;
  if (cudaMemcpyAsync(&b.d_scen[slot].p, &p, sizeof(p), cudaMemcpyHostToDevice, b.cst) !=
          cudaSuccess ||
      cudaMemcpyAsync(b.d_ctl + slot, &h, sizeof(h), cudaMemcpyHostToDevice, b.cst) !=
          cudaSuccess)
    return fail(cuda_fail(cudaGetLastError()));
  // Initial Hmax (src/kernels.cpp:29-34 on the starting state).
  const unsigned gr = grid_for((long long)L.nx * L.ny, 256, 8);
  if (b.prec == AF_PREC_F64)
    k_hmax_int<double><<<gr, 256, 0, b.cst>>>((const double*)p.H[0], (const double*)p.DEM, L.nx,
                                               L.ny, L.P, c->nodata, &p.ctl->hmax_acc);
  else
    k_hmax_int<float><<<gr, 256, 0, b.cst>>>((const float*)p.H[0], (const float*)p.DEM, L.nx,
                                              L.ny, L.P, c->nodata, &p.ctl->hmax_acc);
  k_ctl_fold_hmax<<<1, 1, 0, b.cst>>>(p.ctl);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(b.cst);
  if (e != cudaSuccess) return fail(cuda_fail(e));
  Slot& s = b.slots[slot];
  s.state = 1;
  s.off = off;
  s.L = L;
  s.c = *c;
  s.t_stop = t_stop;
  s.cls = size_class((long long)c->nx * c->ny);
  s.spec = std::move(tb.spec);
  s.p = p;
  b.h_ctl[slot] = h;  // the mirror until the next sync (Hmax not yet read back)
  b.hi_slot = std::max(b.hi_slot, slot + 1);
  b.members_dirty = true;
  *slot_out = slot;
  return AF_OK;
}

static bool finished(const Batch& b, int slot);

// Re-cuts a member into strips of R rows: the strip index of its special
// cells (the cells themselves are in an order that does not depend on R) and
// its parameters.  Results do not depend on R; only the volume diagnostics'
// rounding does.  Stream-ordered before the next launch.
static int set_slot_rows(Batch& b, int slot, int R) {
  Slot& s = b.slots[slot];
  const int own = 30 * b.N;
  const int nsy = (s.L.ny + R - 1) / R;
  const size_t nstrips = (size_t)s.L.nsx * nsy;
  std::vector<int> off(nstrips + 1, 0);
  for (const SpecCell& e : s.spec) off[(size_t)(e.col / own) * nsy + e.row / R + 1]++;
  for (size_t k = 0; k < nstrips; k++) off[k + 1] += off[k];
  char* base = b.arena + s.off;
  AF_CUDA(cudaMemcpyAsync(base + s.L.spec_off, off.data(), off.size() * sizeof(int),
                          cudaMemcpyHostToDevice, b.st));
  s.p.R = R;
  s.p.nsy = nsy;
  s.L.R = R;
  s.L.nsy = nsy;
  AF_CUDA(cudaMemcpyAsync(&b.d_scen[slot].p, &s.p, sizeof(StepParams), cudaMemcpyHostToDevice,
                          b.st));
  // Pageable sources: wait until the copies have left host memory.
  AF_CUDA(cudaStreamSynchronize(b.st));
  return AF_OK;
}

// Load-adaptive strip height: the tuned height of each member's size class,
// lowered (in powers of two, to at least 2 rows) until the active members
// give every warp of the persistent grid about `balance` strips, so the
// steps near the end of a run, when few scenarios remain, keep the SMs busy.
static int retile(Batch& b) {
  if (b.balance <= 0) return AF_OK;
  std::vector<int> act;
  for (int k = 0; k < b.hi_slot; k++)
    if (b.slots[k].state == 1 && !finished(b, k)) act.push_back(k);
  if (act.empty()) return AF_OK;
  const long long target = (long long)b.balance * b.grid.x * b.WY;
  auto units = [&](int Rcap) {
    long long u = 0;
    for (int k : act) {
      const Slot& s = b.slots[k];
      const int R = std::min(b.rows[s.cls], Rcap);
      u += (long long)s.L.nsx * ((s.L.ny + R - 1) / R);
    }
    return u;
  };
  int Rload = 2;
  for (int R = 4096; R >= 2; R >>= 1)
    if (units(R) >= target) {
      Rload = R;
      break;
    }
  for (int k : act) {
    const int R = std::max(1, std::min(b.rows[b.slots[k].cls], Rload));
    if (R != b.slots[k].L.R) AF_TRY(set_slot_rows(b, k, R));
  }
  return AF_OK;
}

static int launch(Batch& b, long long max_steps, int stop_on_done) {
  if (b.in_flight) return AF_ESTATE;
  AF_CUDA(cudaSetDevice(b.device));
  AF_TRY(retile(b));
  if (b.members_dirty) {
    int n = 0;
    for (int k = 0; k < b.hi_slot; k++)
      if (b.slots[k].state == 1) b.h_tab->member[n++] = k;
    b.h_tab->nmember = n;
    AF_CUDA(cudaMemcpyAsync(b.d_tab, b.h_tab, offsetof(BatchTab, member) + sizeof(int) * n,
                            cudaMemcpyHostToDevice, b.st));
    b.members_dirty = false;
  }
  *(volatile int*)b.h_attn = 0;
  if (b.use_cond) {
    void* bargs[] = {&b.bp, &max_steps, &stop_on_done};
    cudaKernelNodeParams kb{};
    kb.func = const_cast<void*>(b.begin_kernel());
    kb.gridDim = dim3(1);
    kb.blockDim = dim3(kFoldThreads);
    kb.kernelParams = bargs;
    AF_CUDA(cudaGraphExecKernelNodeSetParams(b.exec, b.begin_node, &kb));
    AF_CUDA(cudaGraphLaunch(b.exec, b.st));
  } else {
    // Host-driven launches, in batches of 64 steps with a status check.
    BatchParams p = b.bp;
    void* bargs[] = {&p, &max_steps, &stop_on_done};
    AF_CUDA(cudaLaunchKernel(b.begin_kernel(), dim3(1), dim3(kFoldThreads), bargs, 0, b.st));
    void* args[] = {&p};
    long long left = max_steps;
    while (left > 0) {
      const long long n = left < 64 ? left : 64;
      for (long long k = 0; k < n; k++) {
        AF_CUDA(cudaLaunchKernel(b.kernel(), b.grid, b.block, args, 0, b.st));
        AF_CUDA(cudaLaunchKernel(b.fold_kernel(), dim3(1), dim3(kFoldThreads), args, 0, b.st));
      }
      left -= n;
      AF_CUDA(cudaMemcpyAsync(b.h_bctl, b.d_bctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, b.st));
      AF_CUDA(cudaStreamSynchronize(b.st));
      if (b.h_bctl->done) break;
    }
  }
  b.in_flight = true;
  return AF_OK;
}

static int sync(Batch& b) {
  AF_CUDA(cudaSetDevice(b.device));
  AF_CUDA(cudaStreamSynchronize(b.st));
  b.in_flight = false;
  if (b.hi_slot > 0)
    AF_CUDA(cudaMemcpyAsync(b.h_ctl, b.d_ctl, sizeof(SimCtl) * b.hi_slot, cudaMemcpyDeviceToHost,
                            b.st));
  AF_CUDA(cudaMemcpyAsync(b.h_bctl, b.d_bctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, b.st));
  AF_CUDA(cudaStreamSynchronize(b.st));
  for (int k = 0; k < b.hi_slot; k++) {
    Slot& s = b.slots[k];
    if (s.state == 2) {
      b.plan.release(s.off);
      s = Slot();
    }
  }
  return b.h_bctl->status ? AF_ESTATE : AF_OK;
}

static bool finished(const Batch& b, int slot) {
  const SimCtl& c = b.h_ctl[slot];
  return c.status != 0 || !(c.t < c.t_stop) || c.step >= c.step_stop;
}

// A padded field (first element at src) -> caller FP64 rows at host pitch
// hpitch, on the copy stream; FP32 is converted on the device first.
template <typename T>
static int get_field(Batch& b, const char* src, int rows, int width, int P, double* dst,
                     size_t hpitch) {
  if (sizeof(T) == 8) {
    AF_CUDA(copy2d_d2h(dst, hpitch * 8, src, (size_t)P * 8, (size_t)width * 8, rows, b.cst));
  } else {
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(rows, kStageBytes / (8 * (size_t)width)));
    for (int j = 0; j < rows; j += chunk) {
      const int n = std::min(chunk, rows - j);
      k_dense_to_f64<<<grid_for((long long)n * width, 256, 8), 256, 0, b.cst>>>(
          reinterpret_cast<const float*>(src) + (size_t)j * P, P, n, width, b.stage);
      AF_CUDA(cudaGetLastError());
      AF_CUDA(copy2d_d2h(dst + (size_t)j * hpitch, hpitch * 8, b.stage, (size_t)width * 8,
                         (size_t)width * 8, n, b.cst));
    }
  }
  AF_CUDA(cudaStreamSynchronize(b.cst));
  return AF_OK;
}

static int get_state(Batch& b, int slot, double* H, double* Qx, double* Qy) {
  if (slot < 0 || slot >= kMaxSlots || b.slots[slot].state != 1) return AF_EINVAL;
  if (b.in_flight && !finished(b, slot)) return AF_ESTATE;
  AF_CUDA(cudaSetDevice(b.device));
  const Slot& s = b.slots[slot];
  const Layout& L = s.L;
  const int par = b.h_ctl[slot].parity;
  const char* base = b.arena + s.off;
  const size_t g = (size_t)kGuard * b.esize;
  const int nx = L.nx, ny = L.ny;
  auto get = [&](size_t off, int rows, int width, double* dst, size_t hp) {
    return b.prec == AF_PREC_F64 ? get_field<double>(b, base + off + g, rows, width, L.P, dst, hp)
                                 : get_field<float>(b, base + off + g, rows, width, L.P, dst, hp);
  };
  if (H) AF_TRY(get(L.H[par], ny, nx, H, nx));
  if (Qx) {
    AF_TRY(get(L.Qx[par], ny, nx + 1, Qx, nx + 1));
    for (int i = 0; i <= nx; i++) Qx[(size_t)ny * (nx + 1) + i] = 0.0;
  }
  if (Qy) {
    AF_TRY(get(L.Qy[par], ny + 1, nx, Qy, nx + 1));
    for (int j = 0; j <= ny; j++) Qy[(size_t)j * (nx + 1) + nx] = 0.0;
  }
  return AF_OK;
}

}  // namespace af

using af::Batch;

struct af_batch {
  Batch* b;
};

extern "C" {

int af_batch_create(int precision, int device, uint64_t arena_bytes, int variant, af_batch** out) {
  if (!out) return AF_EINVAL;
  Batch* b = nullptr;
  const int rc = af::create(precision, device, arena_bytes, variant, &b);
  if (rc != AF_OK) return rc;
  *out = new af_batch{b};
  return AF_OK;
}

int af_batch_destroy(af_batch* h) {
  if (!h) return AF_EINVAL;
  delete h->b;
  delete h;
  return AF_OK;
}

int af_batch_size_class(int nx, int ny) {
  if (nx < 1 || ny < 1) return AF_EINVAL;
  return af::size_class((long long)nx * ny);
}

int af_batch_set_rows(af_batch* h, int size_class, int rows) {
  if (!h || size_class < 0 || size_class >= af::kClasses || rows < 1 || rows > 4096)
    return AF_EINVAL;
  h->b->rows[size_class] = rows;
  return AF_OK;
}

int af_batch_get_rows(const af_batch* h, int size_class) {
  if (!h || size_class < 0 || size_class >= af::kClasses) return AF_EINVAL;
  return h->b->rows[size_class];
}

int af_batch_footprint(const af_batch* h, const af_case_desc* c, const af_forcing_desc* f,
                       double t_stop, uint64_t* bytes) {
  if (!h || !bytes) return AF_EINVAL;
  AF_TRY(af::check_case(c, f));
  const Batch& b = *h->b;
  const int R = b.rows[af::size_class((long long)c->nx * c->ny)];
  *bytes = af::make_layout(c, f, t_stop, R, b.esize).total;
  return AF_OK;
}

int af_batch_add(af_batch* h, const af_case_desc* c, const af_forcing_desc* f, const double* dem,
                 const double* h0, double t_stop, int* slot) {
  if (!h) return AF_EINVAL;
  return af::add(*h->b, c, f, dem, h0, t_stop, slot);
}

int af_batch_remove(af_batch* h, int slot) {
  if (!h || slot < 0 || slot >= af::kMaxSlots) return AF_EINVAL;
  Batch& b = *h->b;
  af::Slot& s = b.slots[slot];
  if (s.state != 1) return AF_EINVAL;
  b.members_dirty = true;
  if (b.in_flight) {
    s.state = 2;  // released by the next af_batch_sync
    return AF_OK;
  }
  b.plan.release(s.off);
  s = af::Slot();
  return AF_OK;
}

int af_batch_launch(af_batch* h, int64_t max_steps, int stop_on_done) {
  if (!h) return AF_EINVAL;
  return af::launch(*h->b, max_steps, stop_on_done);
}

int af_batch_attention(af_batch* h) {
  if (!h) return AF_EINVAL;
  *(volatile int*)h->b->h_attn = 1;
  return AF_OK;
}

int af_batch_query(af_batch* h) {
  if (!h) return AF_EINVAL;
  Batch& b = *h->b;
  if (!b.in_flight) return 1;
  AF_CUDA(cudaSetDevice(b.device));
  const cudaError_t e = cudaStreamQuery(b.st);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) return 0;
  return af::cuda_fail(e);
}

int af_batch_sync(af_batch* h) {
  if (!h) return AF_EINVAL;
  return af::sync(*h->b);
}

int af_batch_run(af_batch* h, int64_t max_steps, int64_t* batch_steps) {
  if (!h) return AF_EINVAL;
  Batch& b = *h->b;
  const long long before = b.h_bctl->step;
  int rc = AF_OK;
  // With the load-adaptive strip height, each launch ends when a scenario
  // finishes, so the next one is cut for the members that remain.
  for (;;) {
    const long long left = max_steps - (b.h_bctl->step - before);
    if (left <= 0) break;
    AF_TRY(af::launch(b, left, b.balance > 0));
    rc = af::sync(b);
    if (rc != AF_OK) break;
    bool any = false;
    for (int k = 0; k < b.hi_slot && !any; k++)
      any = b.slots[k].state == 1 && !af::finished(b, k);
    if (!any || b.balance <= 0) break;
  }
  if (batch_steps) *batch_steps = b.h_bctl->step - before;
  return rc;
}

int af_batch_set_balance(af_batch* h, int strips_per_warp) {
  if (!h || strips_per_warp < 0) return AF_EINVAL;
  h->b->balance = strips_per_warp;
  return AF_OK;
}

int af_batch_slot_status(const af_batch* h, int slot, double* t, double* dt_last, double* hmax,
                         int64_t* steps, int* state) {
  if (!h || slot < 0 || slot >= af::kMaxSlots) return AF_EINVAL;
  const Batch& b = *h->b;
  if (b.slots[slot].state == 0) return AF_EINVAL;
  const af::SimCtl& c = b.h_ctl[slot];
  if (t) *t = c.t;
  if (dt_last) *dt_last = c.dt_last;
  if (hmax) *hmax = c.hmax;
  if (steps) *steps = c.step;
  if (state) *state = c.status != 0 ? -1 : (af::finished(b, slot) ? 1 : 0);
  return AF_OK;
}

int af_batch_get_state(af_batch* h, int slot, double* H, double* Qx, double* Qy) {
  if (!h) return AF_EINVAL;
  return af::get_state(*h->b, slot, H, Qx, Qy);
}

int af_batch_mass_series(af_batch* h, int slot, double* t, double* vol, double* area, int cap,
                         int* n) {
  if (!h || !n || cap < 0 || slot < 0 || slot >= af::kMaxSlots) return AF_EINVAL;
  Batch& b = *h->b;
  const af::Slot& s = b.slots[slot];
  if (s.state != 1) return AF_EINVAL;
  if (b.in_flight && !af::finished(b, slot)) return AF_ESTATE;
  AF_CUDA(cudaSetDevice(b.device));
  const int cnt = std::min(b.h_ctl[slot].mass_count, cap);
  std::vector<double> buf((size_t)std::max(cnt, 1) * 3);
  if (cnt > 0) {
    AF_CUDA(cudaMemcpyAsync(buf.data(), b.arena + s.off + s.L.mass, (size_t)cnt * 24,
                            cudaMemcpyDeviceToHost, b.cst));
    AF_CUDA(cudaStreamSynchronize(b.cst));
  }
  for (int k = 0; k < cnt; k++) {
    if (t) t[k] = buf[3 * k];
    if (vol) vol[k] = buf[3 * k + 1];
    if (area) area[k] = buf[3 * k + 2];
  }
  *n = b.h_ctl[slot].mass_count;
  return AF_OK;
}

int af_batch_set_trace(af_batch* h, int64_t cap) {
  if (!h || cap < 0) return AF_EINVAL;
  Batch& b = *h->b;
  if (b.in_flight) return AF_ESTATE;
  AF_CUDA(cudaSetDevice(b.device));
  AF_CUDA(cudaStreamSynchronize(b.st));
  if (b.d_trace) {
    AF_CUDA(cudaFree(b.d_trace));
    b.d_trace = nullptr;
  }
  if (cap > 0) AF_TRY(af::alloc_dev((void**)&b.d_trace, (size_t)cap * 32));
  af::BatchCtl& c = *b.h_bctl;
  c.trace = b.d_trace;
  c.trace_base = c.step;
  c.trace_cap = cap;
  const size_t off = offsetof(af::BatchCtl, trace);
  AF_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(b.d_bctl) + off,
                          reinterpret_cast<char*>(&c) + off, sizeof(af::BatchCtl) - off,
                          cudaMemcpyHostToDevice, b.st));
  AF_CUDA(cudaStreamSynchronize(b.st));
  return AF_OK;
}

int af_batch_get_trace(af_batch* h, int64_t* rec, int64_t cap, int64_t* n) {
  if (!h || !n || cap < 0 || (cap > 0 && !rec)) return AF_EINVAL;
  Batch& b = *h->b;
  if (b.in_flight) return AF_ESTATE;
  const af::BatchCtl& c = *b.h_bctl;
  long long have = b.d_trace ? std::min(c.step - c.trace_base, c.trace_cap) : 0;
  if (have < 0) have = 0;
  *n = have;
  const long long k = std::min<long long>(have, cap);
  if (k > 0) {
    AF_CUDA(cudaSetDevice(b.device));
    AF_CUDA(cudaMemcpyAsync(rec, b.d_trace, (size_t)k * 32, cudaMemcpyDeviceToHost, b.st));
    AF_CUDA(cudaStreamSynchronize(b.st));
  }
  return AF_OK;
}

int af_batch_info(const af_batch* h, int* members, int64_t* batch_steps, uint64_t* arena_bytes,
                  uint64_t* arena_used, uint64_t* arena_largest_free) {
  if (!h) return AF_EINVAL;
  const Batch& b = *h->b;
  if (members) {
    int n = 0;
    for (int k = 0; k < b.hi_slot; k++) n += b.slots[k].state == 1;
    *members = n;
  }
  if (batch_steps) *batch_steps = b.h_bctl->step;
  if (arena_bytes) *arena_bytes = b.plan.size();
  if (arena_used) *arena_used = b.plan.used();
  if (arena_largest_free) *arena_largest_free = b.plan.largest_free();
  return AF_OK;
}

void* af_batch_stream(af_batch* h) { return h ? (void*)h->b->st : nullptr; }

}  // extern "C"
