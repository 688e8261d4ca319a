// af_step.cuh -- the fused local-inertial time step (one kernel per step).
//
// One launch performs the whole body of the reference's time loop,
// src/main.cpp:227-288: the CFL time step from the previous state's Hmax
// (src/kernels.cpp:29-43), the interior face fluxes (:46-143), the edge faces
// (:149-256), the point sources (src/main.cpp:245-262), rainfall
// (src/kernels.cpp:354-367), the depth update (:280-290), the point depth
// BCs (:259-277) and the Qold update (:6-19, folded into the loads), and ends
// with the reductions the next step needs (Hmax) and, at mass-report times,
// the volume and flooded area (src/main.cpp:291-304).
//
// Work decomposition ("strips"): a warp owns OWN = 30*N consecutive columns
// and R consecutive rows and marches down the rows.  Its 32 lanes each load N
// consecutive cells (one 16-byte vector: N = 2 doubles or 4 floats) of every
// array; lanes 0 and 31 are halo lanes whose cells belong to the neighbouring
// warps, so every x-neighbour a face needs is one warp shuffle away and the
// warp never touches shared memory.  Each face flux is computed by the lane
// that owns the cell east (x-faces) or south (y-faces) of it, once per step,
// except the face columns at strip edges and the face row above a strip,
// which the neighbouring strip recomputes (identically) instead of waiting.
//
// State is ping-ponged: the step reads buffer `parity` and writes the other.
// The stored fluxes are Q (m^3/s); the reference's Qold = Q*(1/dx) is formed
// when a face is loaded, with the same rounding the reference's UpdateQs
// uses, so no Qold arrays exist.
//
// Control lives in device memory (SimCtl): time, Hmax, parity, step counters.
// The last block to finish (one atomic counter, no waiting) folds Hmax,
// advances time, computes the next step's rain rate and decides whether the
// loop continues (the condition of the enclosing CUDA-graph while node).
#pragma once

#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>
#include <cstdlib>

#include "af_common.cuh"
#include "af_pow.cuh"

// FP32 face-law experiments: AF_FRICTION 1 evaluates the friction factors
// correctly rounded; AF_FACE_FORM 1 forms the flow depth and the head
// difference from surface elevations (2: the flow depth only, 3: the head
// difference only).  Both 0 in the library.
#ifndef AF_FRICTION
#define AF_FRICTION 0
#endif
#ifndef AF_FACE_FORM
#define AF_FACE_FORM 0
#endif
// Batch kernel: 1 hands out units past the first round from a per-step
// counter (dynamic), 0 assigns unit w + k*W to warp w (static).
#ifndef AF_BATCH_DYNAMIC
#define AF_BATCH_DYNAMIC 1
#endif
// FP32 face-law shape: 1 selects the upstream side once per face and forms
// |Qv| hflow^(-7/3) as one exp2 (see flux2).
#ifndef AF_FLUX_V2
#define AF_FLUX_V2 0
#endif
// 1: one lane issues each row's bulk copies (else four lanes, one array each).
#ifndef AF_ISSUE_ONE_LANE
#define AF_ISSUE_ONE_LANE 0
#endif

namespace af {

// Device control block of one simulation.
struct SimCtl {
  double t;           // time at the start of the next step
  double hmax;        // max H over valid cells of the current state
  double dt_last;     // dt of the last step
  double rain_rate;   // rain rate at t (0 without rain)
  double t_stop;      // the loop runs while t < t_stop ...
  double next_mass;   // next mass-report time
  long long step;     // steps taken so far
  long long step_stop;  // ... and step < step_stop
  unsigned long long hmax_acc;  // ordered-bits accumulator of this step's Hmax
  unsigned int arrive;          // blocks (one grid) or strips (batch) finished in this step
  int done;
  int parity;         // buffer holding the current state
  int mass_count;     // entries recorded in the mass series
  int mass_cap;
  int status;
};

// One special cell: a cell that has point sources and/or a point depth BC.
struct SpecCell {
  int row, col;
  int s0, s1;  // sorted-source range (file order within the cell)
  int bc;      // index of the last effective FREE/HFIX/HVAR boundary, or -1
  int pad;
};

// Everything one step needs; passed by value (kernel parameter space).
struct StepParams {
  void* H[2];
  void* Qx[2];
  void* Qy[2];
  const void* DEM;
  int nx, ny, P;      // grid and row pitch (elements)
  int nsx, nsy, R;    // strips in x and y, rows per strip
  double dx, dxinv, dA, fpn, depth_thresh, max_hflow, g, cfl, init_tstep, nodata;
  double mass_int;
  int wf, ef, nf, sf;
  int has_nodata;  // some DEM cell (as stored) equals nodata; 0 lets FP32 skip the tests
  // point sources, sorted by cell (file order within a cell)
  const int* src_type;
  const double* src_value;
  const int* src_off;
  const double* src_times;
  const double* src_vals;
  const unsigned char* src_sorted;
  // point depth BCs (file order)
  const int* bc_type;
  const double* bc_value;
  const int* bc_off;
  const double* bc_times;
  const double* bc_vals;
  const unsigned char* bc_sorted;
  // rain
  const double* rain_times;
  const double* rain_rates;
  int n_rain, rain_sorted;
  // special cells per strip (CSR over strip id = sx*nsy + sy, sorted by row, col)
  const int* spec_off;
  const SpecCell* spec;
  SimCtl* ctl;
  double* partials;     // 3 doubles per block: volume, its compensation, area
  double* mass_series;  // 3 doubles per entry: t, volume, area
  cudaGraphConditionalHandle cond;
  int use_cond;
};

template <typename T>
struct Lanes;
template <>
struct Lanes<double> {
  static constexpr int N = 2;
};
template <>
struct Lanes<float> {
  static constexpr int N = 4;
};

template <typename T>
__device__ inline T gmaxT(T a, T b) { return (a > b) ? a : b; }  // src/types.hpp:14
template <typename T>
__device__ inline T gminT(T a, T b) { return (a < b) ? a : b; }  // src/types.hpp:15

__device__ inline void st_vec(double* p, const double (&v)[2]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}
__device__ inline void st_vec(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

template <typename T>
struct Phys {
  T dx, fn, depth_thresh, max_hflow, nodata, gdt;  // gdt = g*dt
  T g;
  T dxinv, gdt_fn2;  // 1/dx and g*dt*fn*fn/dx (FP32 form only)
};

// FREE edges (src/kernels.cpp:154-248).  West also needs the cell east of
// the edge cell.
template <typename T>
__device__ inline T west_free(T h0, T z0, T h1, T z1, T g, T dx, T nodata) {
  if (z0 == nodata || h0 < T(0.001)) return T(0);
  T y0 = z0 + h0, y1 = z1 + h1;
  if (y0 > z0) {
    T Sf = (y1 - y0) / dx;
    if (Sf < 0) return -h0 * sqrt(g * h0) * dx * T(0.5);
  }
  return T(0);
}
// FP32: the same edge law with the head difference formed from differences
// of close values (see flux2); y0 > z0 is h0 > 0 there.
template <>
__device__ inline float west_free<float>(float h0, float z0, float h1, float z1, float g, float dx,
                                         float nodata) {
  if (z0 == nodata || h0 < 0.001f) return 0.0f;
  if (h0 > 0.0f && (z1 - z0) + (h1 - h0) < 0.0f) return -h0 * sqrtf(g * h0) * dx * 0.5f;
  return 0.0f;
}
template <typename T>
__device__ inline T out_free(T h0, T z0, T sign, T g, T dx, T nodata) {
  if (z0 == nodata || h0 < T(0.001)) return T(0);
  if (h0 > T(0.001)) return sign * h0 * sqrt(g * h0) * dx * T(0.5);
  return T(0);
}

__device__ inline double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline double warp_maxd(double m) {
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_xor_sync(0xffffffffu, m, o);
    if (v > m) m = v;
  }
  return m;
}

// Neumaier-compensated accumulation.
__device__ inline void kahan_add(double& s, double& c, double x) {
  double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x;
  else c += (x - t) + s;
  s = t;
}

// Special-cell helpers (a handful of calls per step) take scalar arguments,
// not the parameter block, so they never force it into local memory.
struct SeriesTable {
  const int* type;
  const double* value;
  const int* off;
  const double* times;
  const double* vals;
  const unsigned char* sorted;
};

// src/main.cpp:246-259 for the sources [s0, s1) of one cell, in file order.
template <typename T>
__device__ inline T apply_sources(T h, int s0, int s1, SeriesTable tb, double dx, double dA,
                                        double t, double dt) {
  for (int s = s0; s < s1; s++) {
    double v;
    if (tb.type[s] == AF_BC_QFIX) {
      v = tb.value[s];
    } else {
      const int o = tb.off[s];
      v = interp_series(tb.times + o, tb.vals + o, tb.off[s + 1] - o, tb.value[s], t,
                        tb.sorted[s] != 0);
    }
    const double ps = v * dx * dt / dA;  // src/main.cpp:253
    h = h + T(ps);
    if (h < T(0)) h = T(0);
  }
  return h;
}

// src/kernels.cpp:266-273 (FREE -> 0, HFIX -> value, HVAR -> value at t).
template <typename T>
__device__ inline T bc_depth(int b, SeriesTable tb, double t) {
  const int ty = tb.type[b];
  if (ty == 1) return T(0);
  if (ty == 2) return T(tb.value[b]);
  const int o = tb.off[b];
  return T(interp_series(tb.times + o, tb.vals + o, tb.off[b + 1] - o, tb.value[b], t,
                         tb.sorted[b] != 0));
}

// ------------------------------------------------------------ row faces
// Interior-formula fluxes of one row for one lane: the west face of each of
// its N cells (qw) and, when `south`, the south face of each (qs).  Inputs are
// the lane's cells of rows j (h, z, qxo, qyo) and j+1 (hN, zN, qxoN, qyoN),
// Qold already formed, and the neighbours from the adjacent lanes (L = the
// cell west of the first, R = the cell east of the last).  The expensive part
// runs only in warps that have a wet face, and there without branches, so the
// faces of a lane overlap in the pipelines.  With theta == 1 the reference's
// `if (Q*dh < 0)` recomputation (src/kernels.cpp:86-89) yields the same Q
// (both numerators are equal whenever Q != 0), so it is not repeated.

// The FP64 wet-face expression out of line (the same results), for the step
// kernel of mid-size grids: the four inline copies per row of a lane make the
// row loop's code large enough to stall on instruction fetch.  Measured, ms
// per step out of line against inline: 724^2 0.0714 / 0.0823, 1024^2 0.106 /
// 0.124, 2048^2 0.247 / 0.269, 4096^2 0.676 / 0.716, 5793^2 1.222 / 1.265;
// level at 512^2 (one wave of strips) and 6896^2, and on 8192^2 inline is
// faster (2.22 against 2.32: the four faces' chains overlap in the FP64 pipe).
static __device__ __noinline__ double face_q64(double dh, double hflow, double q0, double qa, double qb,
                                        double qc, double qd, double dx, double gdt, double fn) {
  const double Sf = -dh / dx;
  const double qy_avg = (qa + qb + qc + qd) / 4.0;
  const double qvect = sqrt(q0 * q0 + qy_avg * qy_avg);
  const double numerator = (q0 + 0.0) - (gdt * hflow * Sf);
  const double denominator =
      1.0 + gdt * hflow * fn * fn * fabs(qvect) / pw::pow_ref(hflow, 10.0 / 3.0);
  return numerator / denominator * dx;
}

// FP64: the reference's expressions exactly (src/kernels.cpp:60-84), with the
// C library's pow algorithm (af_pow.cuh).
template <bool ND, bool kCall = false>  // FP64 keeps every test of the reference
__device__ inline void row_faces(const double (&h)[2], const double (&z)[2], const double (&hN)[2],
                                 const double (&zN)[2], const double (&qxo)[2],
                                 const double (&qxoN)[2], const double (&qyo)[2],
                                 const double (&qyoN)[2], double hL, double zL, double qyoL,
                                 double qyoNL, double qxoR, double qxoNR, bool south,
                                 const Phys<double>& ph, double (&qw)[2], double (&qs)[2]) {
  double Z0[4], H0[4], Z1[4], H1[4], Q0[4], QA[4], QB[4], QC[4], QD[4];
  // faces 0,1: west faces of cells 0,1; faces 2,3: south faces of cells 0,1
  Z0[0] = zL;   H0[0] = hL;   Z1[0] = z[0]; H1[0] = h[0];
  Q0[0] = qxo[0]; QA[0] = qyoL; QB[0] = qyo[0]; QC[0] = qyoNL; QD[0] = qyoN[0];
  Z0[1] = z[0]; H0[1] = h[0]; Z1[1] = z[1]; H1[1] = h[1];
  Q0[1] = qxo[1]; QA[1] = qyo[0]; QB[1] = qyo[1]; QC[1] = qyoN[0]; QD[1] = qyoN[1];
  Z0[2] = z[0]; H0[2] = h[0]; Z1[2] = zN[0]; H1[2] = hN[0];
  Q0[2] = qyoN[0]; QA[2] = qxo[0]; QB[2] = qxo[1]; QC[2] = qxoN[0]; QD[2] = qxoN[1];
  Z0[3] = z[1]; H0[3] = h[1]; Z1[3] = zN[1]; H1[3] = hN[1];
  Q0[3] = qyoN[1]; QA[3] = qxo[1]; QB[3] = qxoR; QC[3] = qxoN[1]; QD[3] = qxoNR;
  double y0[4], y1[4], hf[4];
  bool wet[4];
  bool any = false;
#pragma unroll
  for (int f = 0; f < 4; f++) {
    y0[f] = Z0[f] + H0[f];
    y1[f] = Z1[f] + H1[f];
    double hflow = gmaxT(y0[f], y1[f]) - gmaxT(Z0[f], Z1[f]);
    hflow = gmaxT(hflow, 0.0);
    hflow = gminT(hflow, ph.max_hflow);
    hf[f] = hflow;
    wet[f] = (f < 2 || south) && !(Z0[f] == ph.nodata || Z1[f] == ph.nodata) &&
             hflow > ph.depth_thresh;
    any |= wet[f];
  }
  double Q[4] = {0.0, 0.0, 0.0, 0.0};
  if (__any_sync(0xffffffffu, any)) {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const double dh = y0[f] - y1[f];
      double q;
      if constexpr (kCall) {
        q = face_q64(dh, hf[f], Q0[f], QA[f], QB[f], QC[f], QD[f], ph.dx, ph.gdt, ph.fn);
      } else {
        const double Sf = -dh / ph.dx;
        const double hflow = hf[f];
        const double qy_avg = (QA[f] + QB[f] + QC[f] + QD[f]) / 4.0;
        const double qvect = sqrt(Q0[f] * Q0[f] + qy_avg * qy_avg);
        const double numerator = (Q0[f] + 0.0) - (ph.gdt * hflow * Sf);
        const double denominator =
            1.0 + ph.gdt * hflow * ph.fn * ph.fn * fabs(qvect) / pw::pow_ref(hflow, 10.0 / 3.0);
        q = numerator / denominator * ph.dx;
      }
      Q[f] = wet[f] ? q : 0.0;
    }
  }
  qw[0] = Q[0];
  qw[1] = Q[1];
  qs[0] = Q[2];
  qs[1] = Q[3];
}

// FP32: the same face law on pairs of faces with Blackwell's packed FP32x2
// instructions; the friction term is written g*dt*n^2*|q|*hflow^(-7/3), with
// hflow^(-7/3) = exp2(-7/3 * log2(hflow)) on the special-function unit.
__device__ inline float2 f2(float a, float b) { return make_float2(a, b); }

// ND: the grid has nodata cells, so a face touching one is dry; without ND
// every cell is valid and the tests are skipped (the same results).
template <bool ND>
__device__ inline float2 flux2(float2 z0, float2 h0, float2 z1, float2 h1, float2 q0, float2 qa,
                               float2 qb, float2 qc, float2 qd, bool enable,
                               const Phys<float>& ph, bool& any) {
  // Water-surface elevations y = z + h are never formed: in FP32 their ulp
  // (2-8 um at 16-64 m of elevation) would give a lake at rest spurious
  // surface gradients that drive oscillations in deep, weakly damped water.
  // The head difference y0 - y1 = (z0 - z1) + (h0 - h1) and the flow depth
  // max(y0,y1) - max(z0,z1) = h_up + min(0, z_up - z_down) are the same
  // quantities from differences of close values (exact or nearly so).
  const float2 dz = __fadd2_rn(z0, f2(-z1.x, -z1.y));
#if AF_FACE_FORM == 1 || AF_FACE_FORM == 3
  const float2 dh = __fadd2_rn(__fadd2_rn(z0, h0), f2(-(z1.x + h1.x), -(z1.y + h1.y)));
#else
  const float2 dh = __fadd2_rn(dz, __fadd2_rn(h0, f2(-h1.x, -h1.y)));
#endif
#if AF_FACE_FORM == 1 || AF_FACE_FORM == 2
  // flow depth from surface elevations y = z + h (the reference's form in FP32)
  const float2 hfx = f2(fmaxf(z0.x + h0.x, z1.x + h1.x) - fmaxf(z0.x, z1.x),
                        fmaxf(z0.y + h0.y, z1.y + h1.y) - fmaxf(z0.y, z1.y));
#elif AF_FLUX_V2
  // the upstream cell's depth and its bed's drop to the other cell, selected
  // once, then one packed add (the same values as forming both sides)
  const bool ux = dh.x >= 0.0f, uy = dh.y >= 0.0f;
  const float2 hup = f2(ux ? h0.x : h1.x, uy ? h0.y : h1.y);
  const float2 drop = f2(fminf(0.0f, ux ? dz.x : -dz.x), fminf(0.0f, uy ? dz.y : -dz.y));
  const float2 hfx = __fadd2_rn(hup, drop);
#else
  const float2 hfx = f2(dh.x >= 0.0f ? h0.x + fminf(0.0f, dz.x) : h1.x + fminf(0.0f, -dz.x),
                        dh.y >= 0.0f ? h0.y + fminf(0.0f, dz.y) : h1.y + fminf(0.0f, -dz.y));
#endif
  // The reference clamps the flow depth to [0, MaxHflow] and calls the face
  // wet above DepthThresh; with DepthThresh >= 0 (fill_scalars makes the FP32
  // threshold so) the clamp at 0 only matters for faces that are dry either
  // way, whose values are discarded, so it is not applied.  The wet test is on
  // the unclamped depth, so a NaN depth stays dry as in the reference.
  const float2 hf = f2(fminf(hfx.x, ph.max_hflow), fminf(hfx.y, ph.max_hflow));
  const bool vx = !ND || (z0.x != ph.nodata && z1.x != ph.nodata);
  const bool vy = !ND || (z0.y != ph.nodata && z1.y != ph.nodata);
  const bool wx = enable && vx && hfx.x > ph.depth_thresh;
  const bool wy = enable && vy && hfx.y > ph.depth_thresh;
  any |= wx | wy;
  // In units of the stored Q (= Qold*dx): the reference's
  //   Q = (Qold - g*dt*hflow*Sf) / (1 + g*dt*n^2*|Qvect|/hflow^(10/3)) * dx
  // with Sf = -dh/dx is Q = (Q0 + g*dt*hflow*dh) / (1 + g*dt*n^2/dx*|Qv|*hflow^(-7/3)).
  const float2 a = __fmul2_rn(f2(ph.gdt, ph.gdt), hf);
  const float2 num = __ffma2_rn(a, dh, q0);
  const float2 qavg = __fmul2_rn(__fadd2_rn(__fadd2_rn(qa, qb), __fadd2_rn(qc, qd)),
                                 f2(0.25f, 0.25f));
  const float2 qv2 = __ffma2_rn(q0, q0, __fmul2_rn(qavg, qavg));
#if AF_FRICTION == 1
  // correctly rounded friction factors (a diagnostic form: FP64 pow)
  const float2 qv = f2(__fsqrt_rn(qv2.x), __fsqrt_rn(qv2.y));
  const float2 pw = f2((float)pow((double)hf.x, -7.0 / 3.0), (float)pow((double)hf.y, -7.0 / 3.0));
  const float2 den = __ffma2_rn(__fmul2_rn(f2(ph.gdt_fn2, ph.gdt_fn2), qv), pw, f2(1.0f, 1.0f));
  return f2(wx ? __fdiv_rn(num.x, den.x) : 0.0f, wy ? __fdiv_rn(num.y, den.y) : 0.0f);
#elif AF_FLUX_V2
  // |Qv| * hflow^(-7/3) = 2^(log2(Qv^2)/2 - 7/3 log2(hflow)) on the SFU (Qv = 0
  // gives 2^-inf = 0, a friction-free face, as in the reference)
  const float2 lg = __ffma2_rn(f2(__log2f(qv2.x), __log2f(qv2.y)), f2(0.5f, 0.5f),
                               __fmul2_rn(f2(__log2f(hf.x), __log2f(hf.y)),
                                          f2(-7.0f / 3.0f, -7.0f / 3.0f)));
  const float2 den = __ffma2_rn(f2(ph.gdt_fn2, ph.gdt_fn2), f2(exp2f(lg.x), exp2f(lg.y)),
                                f2(1.0f, 1.0f));
#else
  const float2 qv = f2(sqrtf(qv2.x), sqrtf(qv2.y));
  const float2 pw = f2(exp2f(-7.0f / 3.0f * __log2f(hf.x)), exp2f(-7.0f / 3.0f * __log2f(hf.y)));
  const float2 den = __ffma2_rn(__fmul2_rn(f2(ph.gdt_fn2, ph.gdt_fn2), qv), pw, f2(1.0f, 1.0f));
#endif
  return f2(wx ? __fdividef(num.x, den.x) : 0.0f, wy ? __fdividef(num.y, den.y) : 0.0f);
}

template <bool ND, bool kCall = false>  // kCall: FP64 only
__device__ inline void row_faces(const float (&h)[4], const float (&z)[4], const float (&hN)[4],
                                 const float (&zN)[4], const float (&qxo)[4],
                                 const float (&qxoN)[4], const float (&qyo)[4],
                                 const float (&qyoN)[4], float hL, float zL, float qyoL,
                                 float qyoNL, float qxoR, float qxoNR, bool south,
                                 const Phys<float>& ph, float (&qw)[4], float (&qs)[4]) {
  bool any = false;
  // west faces: (cell k-1, cell k) for k = 0..3
  const float2 w01 = flux2<ND>(f2(zL, z[0]), f2(hL, h[0]), f2(z[0], z[1]), f2(h[0], h[1]),
                           f2(qxo[0], qxo[1]), f2(qyoL, qyo[0]), f2(qyo[0], qyo[1]),
                           f2(qyoNL, qyoN[0]), f2(qyoN[0], qyoN[1]), true, ph, any);
  const float2 w23 = flux2<ND>(f2(z[1], z[2]), f2(h[1], h[2]), f2(z[2], z[3]), f2(h[2], h[3]),
                           f2(qxo[2], qxo[3]), f2(qyo[1], qyo[2]), f2(qyo[2], qyo[3]),
                           f2(qyoN[1], qyoN[2]), f2(qyoN[2], qyoN[3]), true, ph, any);
  // south faces: (cell k row j, cell k row j+1)
  const float2 s01 = flux2<ND>(f2(z[0], z[1]), f2(h[0], h[1]), f2(zN[0], zN[1]), f2(hN[0], hN[1]),
                           f2(qyoN[0], qyoN[1]), f2(qxo[0], qxo[1]), f2(qxo[1], qxo[2]),
                           f2(qxoN[0], qxoN[1]), f2(qxoN[1], qxoN[2]), south, ph, any);
  const float2 s23 = flux2<ND>(f2(z[2], z[3]), f2(h[2], h[3]), f2(zN[2], zN[3]), f2(hN[2], hN[3]),
                           f2(qyoN[2], qyoN[3]), f2(qxo[2], qxo[3]), f2(qxo[3], qxoR),
                           f2(qxoN[2], qxoN[3]), f2(qxoN[3], qxoNR), south, ph, any);
  (void)any;
  qw[0] = w01.x; qw[1] = w01.y; qw[2] = w23.x; qw[3] = w23.y;
  qs[0] = s01.x; qs[1] = s01.y; qs[2] = s23.x; qs[3] = s23.y;
}

// ----------------------------------------------------------- row staging
// Each warp streams its rows through a ring of kStages shared-memory stages.
// One stage holds, for one grid row, the warp's window of 32 lanes x 16 bytes
// (512 bytes) of each of H, DEM, Qx and Qy.  Lane 0 fills a stage with bulk
// copies (cp.async.bulk: the TMA engine's untiled global->shared copy, no
// multicast) that complete on the stage's mbarrier; the lanes wait on it,
// read their 16 bytes, and the stage is refilled kStages rows ahead.  Every
// wait is bounded (kWaitLimit polls); on time-out the warp stops, drains its
// copies in flight (bounded again) and flags the control block.
#ifndef AF_STAGES
#define AF_STAGES 3
#endif

constexpr int kStages = AF_STAGES;  // ring depth (rows in flight per warp, incl. the one in use)
// Code-shape knobs of the fused step (compile time): unroll factor of the row
// loop, and whether x-interior strips get their own copy of the row body
// without per-column edge tests.
#ifndef AF_ROW_UNROLL
#define AF_ROW_UNROLL 1
#endif
#ifndef AF_EDGE_SPLIT
#define AF_EDGE_SPLIT 1
#endif
constexpr int kRowUnroll = AF_ROW_UNROLL;
constexpr int kRowBytes = 512;
constexpr long long kWaitLimit = 1LL << 22;
// Polls a warp spends waiting for a row of its ring before it gives up (the
// drain after a give-up keeps kWaitLimit).  A test build sets it to 0, so
// every such wait runs out at once and the time-out path is exercised without
// a slow or stuck copy.
#ifndef AF_RING_WAIT_LIMIT
#define AF_RING_WAIT_LIMIT (1LL << 22)
#endif
constexpr long long kRingWaitLimit = AF_RING_WAIT_LIMIT;

__device__ inline uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ inline void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
               : "memory");
}
__device__ inline void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ inline void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(b))
      : "memory");
}
// One box of a 3-D tensor (TMA tiled copy, no multicast) into shared memory,
// completing on mbarrier `b`.  `map` is the tensor map's address in kernel
// parameter space; x * element size must be a multiple of 16 bytes.
__device__ inline void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                   uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(b))
      : "memory");
}
__device__ inline bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// True once every lane has seen the phase complete; false after `limit` polls.
__device__ inline bool mbar_wait_warp(uint64_t* b, uint32_t parity,
                                      long long limit = kWaitLimit) {
  for (int i = 0; i < (int)limit; i++) {
    const bool ok = mbar_try_wait(b, parity);
    if (__all_sync(0xffffffffu, ok)) return true;
  }
  return false;
}
__device__ inline void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ inline void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ inline void lds_vec(const unsigned char* p, double (&v)[2]) {
  const double2 t = *reinterpret_cast<const double2*>(p);
  v[0] = t.x;
  v[1] = t.y;
}
__device__ inline void lds_vec(const unsigned char* p, float (&v)[4]) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  v[0] = t.x;
  v[1] = t.y;
  v[2] = t.z;
  v[3] = t.w;
}

template <bool B>
struct BoolC {
  static constexpr bool value = B;
};

// Depth update of a lane's cells: rain (src/kernels.cpp:360-365) then the
// flux divergence (src/kernels.cpp:286-287).  FP64 keeps the reference's
// expressions and order.  FP32 forms the cell's whole increment first,
// rain + (dt/dA)*(flux divergence) (one packed FMA), and rounds it into the
// depth once: adding the same small rain increment to every depth on its own
// would round it the same way in every cell of a binade (a bias in the
// volume), while the flux term differs from cell to cell.  The reference's
// clamp between rain and update has no effect there (rain >= 0, depth >= 0).
template <bool ND>  // FP64 keeps every test of the reference
__device__ inline void update_cells(double (&hn)[2], const double (&qw)[2], const double (&qe)[2],
                                    const double (&qn)[2], const double (&qs)[2],
                                    const double (&z)[2], bool rain_on, double rain_depth,
                                    double dt, double dA, double /*dt_dA*/, double nodata) {
#pragma unroll
  for (int k = 0; k < 2; k++) {
    double v = hn[k];
    if (rain_on && z[k] != nodata) {
      v = v + rain_depth;
      if (v < 0.0) v = 0.0;
    }
    v = v + dt * (qw[k] - qe[k] + qn[k] - qs[k]) / dA;
    if (v < 0.0) v = 0.0;
    hn[k] = v;
  }
}
template <bool ND>
__device__ inline void update_cells(float (&hn)[4], const float (&qw)[4], const float (&qe)[4],
                                    const float (&qn)[4], const float (&qs)[4],
                                    const float (&z)[4], bool rain_on, float rain_depth,
                                    float /*dt*/, float /*dA*/, float dt_dA, float nodata) {
  float rk[4];
#pragma unroll
  for (int k = 0; k < 4; k++) rk[k] = (rain_on && (!ND || z[k] != nodata)) ? rain_depth : 0.0f;
#pragma unroll
  for (int k = 0; k < 4; k += 2) {
    const float2 a = __ffma2_rn(f2(qe[k], qe[k + 1]), f2(-1.0f, -1.0f), f2(qw[k], qw[k + 1]));
    const float2 b = __ffma2_rn(f2(qs[k], qs[k + 1]), f2(-1.0f, -1.0f), f2(qn[k], qn[k + 1]));
    const float2 inc = __ffma2_rn(f2(dt_dA, dt_dA), __fadd2_rn(a, b), f2(rk[k], rk[k + 1]));
    const float2 v = __fadd2_rn(f2(hn[k], hn[k + 1]), inc);
    hn[k] = fmaxf(v.x, 0.0f);
    hn[k + 1] = fmaxf(v.y, 0.0f);
  }
}

// ------------------------------------------------------------ one strip
// Per-step values of one grid, derived from its control block at the start of
// the step.
template <typename T>
struct StepScal {
  double t, dt;
  bool mass, rain_on;
  int parity;
  T rain_depth, dtT, dAT, dxinvT, dt_dA;
  Phys<T> ph;
};

// src/kernels.cpp:36-43: dt from the previous state's Hmax.
__device__ inline double step_dt(const StepParams& p, double hmax_prev) {
  return (hmax_prev > p.depth_thresh) ? p.cfl * p.dx / sqrt(p.g * hmax_prev) : p.init_tstep;
}

// The step's constants of the face law, rain and depth update for dt.
template <typename T>
__device__ inline void fill_scalars(const StepParams& p, double t, double dt, double rate,
                                    double next_mass, int parity, StepScal<T>& s) {
  s.t = t;
  s.dt = dt;
  s.mass = p.mass_int > 0.0 && (t + dt >= next_mass);
  s.rain_on = rate > 0.0;  // src/kernels.cpp:356
  s.parity = parity;
  s.rain_depth = T(rate * dt);
  s.dtT = T(dt);
  s.dAT = T(p.dA);
  s.dxinvT = T(p.dxinv);
  s.dt_dA = T(dt / p.dA);
  s.ph.dx = T(p.dx);
  s.ph.fn = T(p.fpn);
  // FP32: at least 0 (the face law relies on it; a negative threshold makes
  // the reference divide 0 by 0 on dry faces anyway).
  s.ph.depth_thresh = sizeof(T) == 4 ? T(fmax(p.depth_thresh, 0.0)) : T(p.depth_thresh);
  s.ph.max_hflow = T(p.max_hflow);
  s.ph.nodata = T(p.nodata);
  s.ph.g = T(p.g);
  s.ph.gdt = T(p.g * dt);  // (g*dt) rounded once, as the reference's left-to-right product does
  s.ph.dxinv = T(1.0 / p.dx);
  s.ph.gdt_fn2 = T(p.g * dt * p.fpn * p.fpn * p.dxinv);
}

template <typename T>
__device__ inline void step_scalars(const StepParams& p, double t, double hmax_prev, double rate,
                                    double next_mass, int parity, StepScal<T>& s) {
  fill_scalars(p, t, step_dt(p, hmax_prev), rate, next_mass, parity, s);
}

// What one lane carries out of its strips: the max depth over its valid
// cells (state precision; exact; -FLT_MAX while it has seen none: depths of
// valid cells are finite and far above it) and, at mass-report steps, its
// volume and flooded-area sums.
// A warp's position in its stage ring: the stage it consumes next and the
// mbarrier phase that stage completes with.  Kept as running counters (the
// ring depth is 3, so deriving them from a stage count would divide by 3).
// Packed in one register: bits 0-1 the slot, bit 2 the phase.
struct RingPos {
  uint32_t v;
  __device__ __forceinline__ int slot() const { return (int)(v & 3u); }
  __device__ __forceinline__ uint32_t phase() const { return v >> 2; }
  __device__ __forceinline__ void advance() {
    v = ((v & 3u) == (uint32_t)(kStages - 1)) ? ((v & 4u) ^ 4u) : v + 1u;
  }
};
static_assert(kStages <= 4, "the ring position packs the slot in two bits");

template <typename T>
struct LaneAcc {
  T m_cell;
  double v, a;
  __device__ bool any_cell() const { return m_cell != T(-FLT_MAX); }
};

// One step of strip (sx, sy) of one grid by one warp: the strip's OWN
// columns and R rows, streamed through the warp's stage ring (`ring`, `bar`;
// `pos` = the warp's position in the ring, advanced past the strip's stages).
// Warps whose strip lies wholly inside the grid in x take a path without the
// per-column edge tests.  Returns false after a wait time-out, with the
// copies in flight drained and the grid's status flagged.
// kSplitND: FP32 grids without nodata cells take a copy of the row loop
// without the nodata tests (the same results; the batch kernel uses it, the
// single-grid kernel measured no faster with it).  kCall: FP64 evaluates each
// wet face out of line (see face_q64).
// kTma: one tiled copy per row through `tmap` instead of four bulk copies.
template <typename T, bool kSplitND = false, bool kCall = false, bool kTma = false>
__device__ __forceinline__ bool run_strip(const StepParams& p, const StepScal<T>& sc, int sx,
                                          int sy, unsigned char (*ring)[4][kRowBytes],
                                          uint64_t* bar, RingPos& pos, LaneAcc<T>& acc,
                                          const CUtensorMap* tmap = nullptr) {
  constexpr int N = Lanes<T>::N;
  constexpr int OWN = 30 * N;
  static_assert(32 * N * sizeof(T) == kRowBytes, "one 16-byte vector per lane");
  // FP64 forms the reference's Qold = Q*(1/dx) on load (its exact rounding);
  // the FP32 face law works on Q itself (1/dx folded into its coefficients).
  constexpr bool kQold = Lanes<T>::N == 2;
  const int lane = threadIdx.x & 31;
  const int nx = p.nx, ny = p.ny, P = p.P;
  const int parity = sc.parity;
  const double t = sc.t, dt = sc.dt;
  const bool mass = sc.mass, rain_on = sc.rain_on;
  const T rain_depth = sc.rain_depth, dtT = sc.dtT, dAT = sc.dAT, dxinvT = sc.dxinvT,
          dt_dA = sc.dt_dA;
  const Phys<T> ph = sc.ph;
  const T* __restrict__ H = static_cast<const T*>(p.H[parity]);
  T* __restrict__ Hn = static_cast<T*>(p.H[parity ^ 1]);
  const T* __restrict__ Qx = static_cast<const T*>(p.Qx[parity]);
  T* __restrict__ Qxn = static_cast<T*>(p.Qx[parity ^ 1]);
  const T* __restrict__ Qy = static_cast<const T*>(p.Qy[parity]);
  T* __restrict__ Qyn = static_cast<T*>(p.Qy[parity ^ 1]);
  const T* __restrict__ Z = static_cast<const T*>(p.DEM);
  bool failed = false;

  const int x0 = sx * OWN;
  const int cb = x0 - N + lane * N;          // first column of this lane
  const long long wcol = (long long)x0 - N;  // first column of the warp's window
  const bool own = lane >= 1 && lane <= 30;
  const int j0 = sy * p.R;
  const int j1 = min(j0 + p.R, ny);
  const int strip = sx * p.nsy + sy;  // column-major: the special-cell order is R-independent
  int sp = p.spec_off[strip];
  const int sp_end = p.spec_off[strip + 1];
  // Row of the strip's next special cell (INT_MAX: none left), loaded as soon
  // as the previous one is consumed, so the row loop's test waits on nothing.
  int next_row = sp < sp_end ? p.spec[sp].row : INT_MAX;
  // Rows to stream: j0-1 (H, DEM, Qx: the prologue) if j0 > 0, then j0..j1
  // (all four; row ny only exists for Qy).
  const int rfirst = j0 > 0 ? j0 - 1 : j0;
  const int nload = j1 + 1 - rfirst;
  // Bytes of each row copy: the whole window, or on a grid's last strip in x
  // the columns up to nx (Qx's east edge face) rounded up to 16 bytes, so the
  // padding past the grid is not read.  The lanes past it see stale stage
  // bytes; every result of theirs is masked (stores, Hmax, volume), and the
  // last valid lane's right-hand neighbour values (Qx at column nx) are copied.
  const uint32_t row_bytes = (uint32_t)min(
      (long long)kRowBytes, (((long long)nx + 1 - wcol) * (long long)sizeof(T) + 15) & ~15LL);
  // Lanes 0..3 each copy one array (H, DEM, Qx, Qy) of row rfirst+k into
  // stage k; lane 0 also posts the expected byte count.  The prologue row
  // j0-1 has no Qy; row ny has only Qy.
#if AF_ISSUE_ONE_LANE
  // Lane 0 issues the row's copies (straight-line code, no per-lane
  // serialisation of the copy instruction); the warp's reads of the stage
  // being refilled are ordered before them by the __syncwarp in release().
  auto issue = [&](int k, int slot) {
    const int r = rfirst + k;
    if (lane == 0) {
      const int a_lo = r < ny ? 0 : 3;
      const int a_hi = r < j0 ? 3 : 4;
      const long long off = (long long)r * P + wcol;
      mbar_expect_tx(&bar[slot], (uint32_t)(a_hi - a_lo) * row_bytes);
      fence_proxy_async();
      if (a_lo == 0) {
        bulk_g2s(&ring[slot][0][0], H + off, row_bytes, &bar[slot]);
        bulk_g2s(&ring[slot][1][0], Z + off, row_bytes, &bar[slot]);
        bulk_g2s(&ring[slot][2][0], Qx + off, row_bytes, &bar[slot]);
      }
      if (a_hi == 4) bulk_g2s(&ring[slot][3][0], Qy + off, row_bytes, &bar[slot]);
    }
  };
#else
  const T* const my_src = lane == 0 ? H : lane == 1 ? Z : lane == 2 ? Qx : Qy;
  auto issue = [&](int k, int slot) {
    const int r = rfirst + k;
    if constexpr (kTma) {
      // One tiled copy of the row's window from all four fields: the fields
      // are planes 4*parity .. 4*parity+3 (H, DEM, Qx, Qy) of one 3-D
      // tensor, so the box {window, 1 row, 4 planes} lands as the stage's
      // four 512-byte rows.  Columns past the grid (and the window's first
      // lane on the west edge) are outside the tensor and read as zeros.
      if (lane == 0) {
        mbar_expect_tx(&bar[slot], 4u * kRowBytes);
        fence_proxy_async();
        tma_load_3d(&ring[slot][0][0], tmap, (int)wcol, r, 4 * parity, &bar[slot]);
      }
    } else {
      const int a_lo = r < ny ? 0 : 3;
      const int a_hi = r < j0 ? 3 : 4;
      if (lane == 0) mbar_expect_tx(&bar[slot], (uint32_t)(a_hi - a_lo) * row_bytes);
      if (lane >= a_lo && lane < a_hi) {
        fence_proxy_async();
        bulk_g2s(&ring[slot][lane][0], my_src + (long long)r * P + wcol, row_bytes, &bar[slot]);
      }
    }
  };
#endif
  {
    RingPos f = pos;
    for (int k = 0; k < kStages && k < nload; k++) {
      issue(k, f.slot());
      f.advance();
    }
  }
  __syncwarp();
  int kc = 0;  // next stage of this strip to consume, at ring position `pos`
  auto acquire = [&]() -> const unsigned char* {
    if (!mbar_wait_warp(&bar[pos.slot()], pos.phase(), kRingWaitLimit)) return nullptr;
    return &ring[pos.slot()][0][0] + lane * 16;
  };
  // The consumed stage is refilled with the row kStages ahead (same slot).
  auto release = [&]() {
    __syncwarp();
    if (kc + kStages < nload) issue(kc + kStages, pos.slot());
    kc++;
    pos.advance();
  };

  T h[N], z[N], qxo[N], qyo[N], qyn[N];
  T hp[N], zp[N], qxp[N];
  if (j0 > 0) {
    const unsigned char* st = acquire();
    if (!st) failed = true;
    if (!failed) {
      lds_vec(st, hp);
      lds_vec(st + kRowBytes, zp);
      lds_vec(st + 2 * kRowBytes, qxp);
      release();
    }
  }
  if (!failed) {
    const unsigned char* st = acquire();
    if (!st) failed = true;
    if (!failed) {
      lds_vec(st, h);
      lds_vec(st + kRowBytes, z);
      lds_vec(st + 2 * kRowBytes, qxo);
      lds_vec(st + 3 * kRowBytes, qyo);
      release();
#pragma unroll
      for (int k = 0; k < N; k++) {
        if (kQold) {
          qxo[k] = qxo[k] * dxinvT;
          qyo[k] = qyo[k] * dxinvT;
        }
      }
    }
  }
  if (!failed) {
    // North faces of row j0.
    if (j0 == 0) {
#pragma unroll
      for (int k = 0; k < N; k++) qyn[k] = p.nf ? out_free(h[k], z[k], T(-1), ph.g, ph.dx, ph.nodata) : T(0);
      if (own) {
        if (cb + N <= nx) {
          st_vec(Qyn + cb, qyn);
        } else {
#pragma unroll
          for (int k = 0; k < N; k++)
            if (cb + k < nx) Qyn[cb + k] = qyn[k];
        }
      }
    } else {
      // The south faces of row j0-1, by the same code (row_faces) that the
      // strip above uses to compute and store them, so both strips see the
      // same flux through their common edge, bit for bit, in either
      // precision.  The west faces it also returns are not needed here.
#pragma unroll
      for (int k = 0; k < N; k++)
        if (kQold) qxp[k] = qxp[k] * dxinvT;
      const T qxpR = __shfl_down_sync(0xffffffffu, qxp[0], 1);
      const T qxoR = __shfl_down_sync(0xffffffffu, qxo[0], 1);
      T qw_unused[N];
      row_faces<true>(hp, zp, h, z, qxp, qxo, qyo, qyo, T(0), T(0), T(0), T(0), qxpR, qxoR, true,
                      ph, qw_unused, qyn);
    }
  }

  auto rows = [&](auto edge_tag, auto nd_tag, auto call_tag) {
    constexpr bool kEdge = decltype(edge_tag)::value;
    constexpr bool kND = decltype(nd_tag)::value;
    constexpr bool kFaceCall = decltype(call_tag)::value;
#pragma unroll kRowUnroll
    for (int j = j0; j < j1; j++) {
      const bool has_next = (j + 1 < ny);
      T hN[N], zN[N], qxoN[N], qyoN[N];
      {
        const unsigned char* st = acquire();
        if (!st) {
          failed = true;
          return;
        }
        lds_vec(st + 3 * kRowBytes, qyoN);
        if (has_next) {
          lds_vec(st, hN);
          lds_vec(st + kRowBytes, zN);
          lds_vec(st + 2 * kRowBytes, qxoN);
        } else {
#pragma unroll
          for (int k = 0; k < N; k++) hN[k] = zN[k] = qxoN[k] = T(0);
        }
        release();
#pragma unroll
        for (int k = 0; k < N; k++) {
          if (kQold) {
            qyoN[k] = qyoN[k] * dxinvT;
            qxoN[k] = qxoN[k] * dxinvT;
          }
        }
      }
      // Neighbours across lanes.
      const T hL = __shfl_up_sync(0xffffffffu, h[N - 1], 1);
      const T zL = __shfl_up_sync(0xffffffffu, z[N - 1], 1);
      const T qyoL = __shfl_up_sync(0xffffffffu, qyo[N - 1], 1);
      const T qyoNL = __shfl_up_sync(0xffffffffu, qyoN[N - 1], 1);
      const T qxoR = __shfl_down_sync(0xffffffffu, qxo[0], 1);
      const T qxoNR = __shfl_down_sync(0xffffffffu, qxoN[0], 1);

      // Faces of the row: interior law everywhere, then the edges.
      T qw[N], qs[N];
      row_faces<kND, kFaceCall>(h, z, hN, zN, qxo, qxoN, qyo, qyoN, hL, zL, qyoL, qyoNL, qxoR,
                                qxoNR,
                     has_next, ph, qw, qs);
      if (kEdge) {
#pragma unroll
        for (int k = 0; k < N; k++) {
          const int c = cb + k;
          if (c == 0) qw[k] = p.wf ? west_free(h[0], z[0], h[1], z[1], ph.g, ph.dx, ph.nodata) : T(0);
          else if (c >= nx) qw[k] = T(0);
        }
      }
      if (!has_next) {
#pragma unroll
        for (int k = 0; k < N; k++) qs[k] = p.sf ? out_free(h[k], z[k], T(1), ph.g, ph.dx, ph.nodata) : T(0);
      }
      const T qwR = __shfl_down_sync(0xffffffffu, qw[0], 1);
      // East face of every cell.
      T qe[N];
#pragma unroll
      for (int k = 0; k < N; k++) qe[k] = (k < N - 1) ? qw[k + 1] : qwR;
      T qe_last = T(0);
      if (kEdge) {
#pragma unroll
        for (int k = 0; k < N; k++) {
          if (cb + k == nx - 1) {
            qe[k] = p.ef ? out_free(h[k], z[k], T(1), ph.g, ph.dx, ph.nodata) : T(0);
            qe_last = qe[k];
          }
        }
      }
      // Depth update of the owned cells.
      T hn[N];
#pragma unroll
      for (int k = 0; k < N; k++) hn[k] = h[k];
      const int sp_row = sp;
      // Point sources (src/main.cpp:245-262), before rain and the update.
      while (next_row == j) {
        const SpecCell e = p.spec[sp];
        const int kc = e.col - cb;  // the lane's cell index of the special cell
        if (own && kc >= 0 && kc < N) {
          // One call site for the lane's N cells (selected, not indexed, so
          // the cells stay in registers): keeps the row loop's code small.
          T hv = hn[0];
#pragma unroll
          for (int k = 1; k < N; k++)
            if (kc == k) hv = hn[k];
          hv = apply_sources(hv, e.s0, e.s1,
                             SeriesTable{p.src_type, p.src_value, p.src_off, p.src_times,
                                         p.src_vals, p.src_sorted},
                             p.dx, p.dA, t, dt);
#pragma unroll
          for (int k = 0; k < N; k++)
            if (kc == k) hn[k] = hv;
        }
        sp++;
        next_row = sp < sp_end ? p.spec[sp].row : INT_MAX;
      }
      update_cells<kND>(hn, qw, qe, qyn, qs, z, rain_on, rain_depth, dtT, dAT, dt_dA, ph.nodata);
      // Point depth BCs (src/kernels.cpp:259-277), after the update.
      for (int q = sp_row; q < sp; q++) {
        const SpecCell e = p.spec[q];
        if (own && e.bc >= 0) {
          const T v = bc_depth<T>(e.bc,
                                  SeriesTable{p.bc_type, p.bc_value, p.bc_off, p.bc_times,
                                              p.bc_vals, p.bc_sorted},
                                  t);
#pragma unroll
          for (int k = 0; k < N; k++)
            if (cb + k == e.col) hn[k] = v;
        }
      }
      if (own) {
        const long long r = (long long)j * P + cb;
        const long long rs = r + P;
        if (!kEdge || cb + N <= nx) {
          st_vec(Hn + r, hn);
          st_vec(Qxn + r, qw);
          st_vec(Qyn + rs, qs);
        } else {
#pragma unroll
          for (int k = 0; k < N; k++) {
            if (cb + k < nx) {
              Hn[r + k] = hn[k];
              Qxn[r + k] = qw[k];
              Qyn[rs + k] = qs[k];
            }
          }
        }
        if (kEdge && cb <= nx - 1 && nx - 1 < cb + N) Qxn[(long long)j * P + nx] = qe_last;
        // Hmax over valid cells (a NaN never wins the comparison).
#pragma unroll
        for (int k = 0; k < N; k++)
          if ((!kEdge || cb + k < nx) && (!kND || z[k] != ph.nodata))
            acc.m_cell = (hn[k] > acc.m_cell) ? hn[k] : acc.m_cell;
        if (__builtin_expect(mass, 0)) {  // warp-uniform: mass-report steps only
#pragma unroll
          for (int k = 0; k < N; k++) {
            if (!kEdge || cb + k < nx) {
              const double hv = (double)hn[k];
              acc.v += hv * p.dA;
              if (hv > 0.01) acc.a += p.dA;
            }
          }
        }
      }
      // Advance one row.
#pragma unroll
      for (int k = 0; k < N; k++) {
        h[k] = hN[k];
        z[k] = zN[k];
        qxo[k] = qxoN[k];
        qyo[k] = qyoN[k];
        qyn[k] = qs[k];
      }
    }
  };
  if (!failed) {
    // FP32 takes a copy of the row loop without nodata tests on grids that
    // have no nodata cell; FP64 keeps the reference's tests everywhere.
    bool nd = true;
    if constexpr (sizeof(T) == 4 && kSplitND) nd = p.has_nodata != 0;
#if AF_EDGE_SPLIT
    const bool interior = (x0 > 0) && (x0 + OWN < nx);
#else
    const bool interior = false;
#endif
    if (nd) {
      if (interior) rows(BoolC<false>(), BoolC<true>(), BoolC<kCall>());
      else rows(BoolC<true>(), BoolC<true>(), BoolC<kCall>());
    } else {
      if constexpr (kSplitND) {
        if (interior) rows(BoolC<false>(), BoolC<false>(), BoolC<false>());
        else rows(BoolC<true>(), BoolC<false>(), BoolC<false>());
      }
    }
  }
  if (failed) {
    // Drain the copies still in flight into this warp's stages (bounded),
    // then flag the control block so the loop stops with an error.
    const int issued = min(nload, kc + kStages);
    RingPos d = pos;
    for (int k = kc; k < issued; k++) {
      mbar_wait_warp(&bar[d.slot()], d.phase());
      d.advance();
    }
    for (int k = kc; k < nload; k++) pos.advance();  // past the strip's stages
    if (lane == 0) atomicExch(&p.ctl->status, 2);
  }
  return !failed;
}

// Folds a finished step into the grid's control block (one thread): the new
// Hmax, t += dt (src/main.cpp:287), the mass report (:291-304), the next
// step's rain rate, and the loop test of :227.  Returns whether this grid's
// loop stops here.
__device__ inline bool fold_step(const StepParams& p, SimCtl* ctl, double t, double dt, int parity,
                                 bool mass, double vol, double area) {
  const unsigned long long acc = atomicExch(&ctl->hmax_acc, ord_encode(-DBL_MAX));
  const double hmax = ord_decode(acc);
  const double t_new = t + dt;  // src/main.cpp:287
  const long long step_new = ctl->step + 1;
  ctl->hmax = hmax;
  ctl->t = t_new;
  ctl->dt_last = dt;
  ctl->step = step_new;
  ctl->parity = parity ^ 1;
  if (mass) {  // src/main.cpp:291-304
    const int k = ctl->mass_count;
    if (k < ctl->mass_cap) {
      p.mass_series[3 * k] = t_new;
      p.mass_series[3 * k + 1] = vol;
      p.mass_series[3 * k + 2] = area;
      ctl->mass_count = k + 1;
    }
    ctl->next_mass += p.mass_int;
  }
  ctl->rain_rate = p.n_rain > 0 ? interp_series(p.rain_times, p.rain_rates, p.n_rain, 0.0, t_new,
                                                p.rain_sorted != 0)
                                : 0.0;
  // A non-positive or non-finite dt (a diverged state) would stall time:
  // stop the loop and report it instead.
  const bool bad = !(dt > 0.0) || !(t_new < 1.0e300) || !(hmax == hmax) ||
                   *(volatile int*)&ctl->status != 0;
  if (bad) ctl->status = 1;
  const bool done = bad || !(t_new < ctl->t_stop) || step_new >= ctl->step_stop;
  ctl->done = done;
  ctl->arrive = 0u;
  return done;
}

// ------------------------------------------------------- single grid
// Persistent grid: block b processes tiles b, b + gridDim.x, ...; a tile is
// WY strips stacked along y (warp w owns strip sy = tile_y*WY + w of column
// strip sx).  The last block to finish folds the step.  kTma: rows are read
// with one tiled copy per row through the tensor map `fields` (the grid's
// fields as planes of one 3-D tensor); otherwise four bulk copies per row.
template <typename T, int WY, int MINB, bool kCall = false, bool kTma = true>
__global__ void __launch_bounds__(32 * WY, MINB) k_step(const StepParams p,
                                                        const __grid_constant__ CUtensorMap fields) {
  __shared__ __align__(128) unsigned char s_ring[WY][kStages][4][kRowBytes];
  __shared__ __align__(8) uint64_t s_bar[WY][kStages];
  SimCtl* ctl = p.ctl;
  if (*(volatile int*)&ctl->done) return;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  StepScal<T> sc;
  step_scalars(p, ctl->t, ctl->hmax, ctl->rain_rate, ctl->next_mass, ctl->parity, sc);
  const bool mass = sc.mass;
  uint64_t* bar = s_bar[warp];
  if (lane == 0) {
    for (int s = 0; s < kStages; s++) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncwarp();
  RingPos pos{0u};
  LaneAcc<T> acc{T(-FLT_MAX), 0.0, 0.0};
  const int tiles_y = (p.nsy + WY - 1) / WY;
  const int ntiles = p.nsx * tiles_y;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int sx = tile % p.nsx;
    const int sy = (tile / p.nsx) * WY + warp;
    if (sy >= p.nsy) continue;
    if (!run_strip<T, false, kCall, kTma>(p, sc, sx, sy, s_ring[warp], bar, pos, acc, &fields))
      break;
  }

  // A valid cell's depth is finite (NaN never wins a comparison), and in
  // FP64 m_cell is exact; a lane with no valid cell keeps the identity.
  double m_loc = -DBL_MAX, v_loc = acc.v, a_loc = acc.a;
  if (acc.any_cell() && (double)acc.m_cell > m_loc) m_loc = (double)acc.m_cell;

  // ----- block reductions: Hmax, and volume/area at mass-report steps -----
  __shared__ double s_m[WY], s_v[WY], s_a[WY];
  __shared__ bool s_last;
  m_loc = warp_maxd(m_loc);
  if (mass) {
    v_loc = warp_sum(v_loc);
    a_loc = warp_sum(a_loc);
  }
  if (lane == 0) {
    s_m[warp] = m_loc;
    s_v[warp] = v_loc;
    s_a[warp] = a_loc;
  }
  __syncthreads();
  const unsigned nblocks = gridDim.x * gridDim.y;
  const unsigned bid = blockIdx.y * gridDim.x + blockIdx.x;
  if (threadIdx.x == 0) {
    double m = s_m[0], v = s_v[0], a = s_a[0];
    for (int w = 1; w < WY; w++) {
      if (s_m[w] > m) m = s_m[w];
      v += s_v[w];
      a += s_a[w];
    }
    if (m > -DBL_MAX) atomicMax(&ctl->hmax_acc, ord_encode(m));
    if (mass) {
      p.partials[3 * bid] = v;
      p.partials[3 * bid + 1] = 0.0;
      p.partials[3 * bid + 2] = a;
    }
    __threadfence();
    unsigned prev = atomicAdd(&ctl->arrive, 1u);
    s_last = (prev == nblocks - 1);
  }
  __syncthreads();
  if (!s_last) return;

  // ----- last block: fold the step into the control block -----
  __threadfence();
  __shared__ double r_v[32 * WY], r_c[32 * WY], r_a[32 * WY];
  if (mass) {
    double s = 0.0, c = 0.0, a = 0.0;
    for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x) {
      kahan_add(s, c, __ldcg(&p.partials[3 * b]));
      a += __ldcg(&p.partials[3 * b + 2]);
    }
    r_v[threadIdx.x] = s;
    r_c[threadIdx.x] = c;
    r_a[threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double S = 0.0, Cc = 0.0, A = 0.0;
      for (int k = 0; k < (int)blockDim.x; k++) {
        kahan_add(S, Cc, r_v[k]);
        Cc += r_c[k];
        A += r_a[k];
      }
      r_v[0] = S + Cc;
      r_a[0] = A;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const bool done = fold_step(p, ctl, sc.t, sc.dt, sc.parity, mass, r_v[0], r_a[0]);
    __threadfence();
    if (p.use_cond) cudaGraphSetConditional(p.cond, done ? 0u : 1u);
  }
}

// ------------------------------------------------------------ batches
// A batch advances many independent grids ("scenarios": each with its own
// size, parameters, forcing, dt and time) by one step each per batch step.
// A batch step is two kernels, and the body of the graph's while loop holds
// kStepsPerIteration batch steps in a row:
//   k_batch_step: the strips of every active scenario.  Units are numbered
//     scenario after scenario (u0[a] = first unit of active scenario a); warp
//     w of the persistent grid takes units w, w + W, ...; within a scenario,
//     unit k is strip (k % nsx, k / nsx), so the warps running at the same
//     time read adjacent 512-byte segments of the same rows.  A unit ends
//     with a fire-and-forget atomicMax of its Hmax and, at mass-report steps,
//     a store of its volume partials; nothing waits.
//     A warp fetches the record of its next unit's scenario (one bulk copy
//     into the second of its two record buffers) while it runs the current
//     unit, so switching scenarios between units costs no wait.
//   k_batch_fold (one block): folds every active scenario's step (a thread
//     per scenario; a warp per volume sum at mass-report steps), writes the
//     scenario's next dt, time, parity and step constants beside its
//     parameters, rebuilds the active list when a scenario has finished, and
//     sets the loop condition.
// A scenario's results do not depend on which other scenarios share the
// batch: every face and cell is computed by the same code, Hmax is an exact
// max, and its volume partials are summed per strip in strip order.
constexpr int kMaxSlots = 1024;
constexpr int kFoldThreads = 1024;  // one block of the fold and begin kernels
// Steps per iteration of a graph's while loop (single grid and batch): the
// loop test runs once per iteration; steps after the one that ends the loop
// return at once (the step and fold kernels check `done` first).
constexpr int kStepsPerIteration = 4;

// Per slot: the scenario's parameters and its coming step.  Copied whole
// into shared memory by one bulk copy (16-byte size and alignment).
struct __align__(16) BatchScen {
  StepParams p;
  double t, dt, rate, next_mass;  // written by the begin and fold kernels
  int parity, pad;
  // The coming step's StepScal<T> (T: the batch's precision), written with t.
  __align__(16) unsigned char scal[sizeof(StepScal<double>)];
};
static_assert(sizeof(BatchScen) % 16 == 0, "bulk-copied record");
static_assert(sizeof(StepScal<float>) <= sizeof(StepScal<double>), "scalar storage");

struct BatchTab {
  int nmember;                // slots in the batch (written by the host)
  int member[kMaxSlots];
  int nact;                   // scenarios stepped by the coming step
  int units;                  // their strips
  long long cells;            // their cells
  int act[kMaxSlots];         // their slots
  int u0[kMaxSlots + 1];      // first unit of each; u0[nact] = units
};

struct BatchCtl {
  long long step;       // batch steps taken
  long long step_stop;  // the loop stops when step reaches this,
  int completed;        // or, with stop_on_done, once a scenario has finished,
  int stop_on_done;
  int done;             // or when nothing is active or the host asks for attention
  int status;           // nonzero: a wait timed out; the batch's state is invalid
  unsigned int next_unit;  // units of the coming step handed out past the first round
  int pad_;
  // Optional per-step trace (af_batch_set_trace): record k describes batch
  // step trace_base + k as {start, end} on the device clock (ns) and the
  // cells and strips it stepped.  Written by the host between launches.
  unsigned long long* trace;
  long long trace_base, trace_cap;
  unsigned long long last_stamp;  // end of the previous step, or the launch's start
};

__device__ inline unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct BatchParams {
  BatchScen* scen;                 // per slot
  BatchTab* tab;
  BatchCtl* bctl;
  const volatile int* attention;   // host memory mapped into the device; may be null
  cudaGraphConditionalHandle cond;
  int use_cond;
};

// The active list: members whose time is below their stop time and whose
// state is sound, with their strip offsets.  One warp.
__device__ inline void batch_compact(const BatchParams& bp) {
  BatchTab* tab = bp.tab;
  const int lane = threadIdx.x & 31;
  const int nm = tab->nmember;
  int nact = 0, units = 0;
  long long cells = 0;
  for (int base = 0; base < nm; base += 32) {
    const int i = base + lane;
    int slot = -1, nu = 0;
    bool act = false;
    if (i < nm) {
      slot = tab->member[i];
      const StepParams* sp = &bp.scen[slot].p;
      const SimCtl* c = sp->ctl;
      act = __ldcg(&c->status) == 0 && __ldcg(&c->t) < __ldcg(&c->t_stop) &&
            __ldcg(&c->step) < __ldcg(&c->step_stop);
      nu = sp->nsx * sp->nsy;
      if (act) cells += (long long)sp->nx * sp->ny;
    }
    const unsigned m = __ballot_sync(0xffffffffu, act);
    int x = act ? nu : 0;  // inclusive scan of the active lanes' strip counts
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (act) {
      const int pos = nact + __popc(m & ((1u << lane) - 1u));
      tab->act[pos] = slot;
      tab->u0[pos] = units + x - nu;
    }
    nact += __popc(m);
    units += __shfl_sync(0xffffffffu, x, 31);
  }
  for (int o = 16; o > 0; o >>= 1) cells += __shfl_xor_sync(0xffffffffu, cells, o);
  if (lane == 0) {
    tab->nact = nact;
    tab->units = units;
    tab->cells = cells;
    tab->u0[nact] = units;
  }
}

// The coming step of one scenario, from its control block, and its constants.
template <typename T>
__device__ inline void batch_next(BatchScen* s) {
  const SimCtl* c = s->p.ctl;
  s->t = c->t;
  s->dt = step_dt(s->p, c->hmax);
  s->rate = c->rain_rate;
  s->next_mass = c->next_mass;
  s->parity = c->parity;
  fill_scalars(s->p, s->t, s->dt, s->rate, s->next_mass, s->parity,
               *reinterpret_cast<StepScal<T>*>(s->scal));
}

// Sets up one launch of the batch loop: the step limit, the active list,
// each active scenario's coming step, and the loop condition.
template <typename T>
__global__ void __launch_bounds__(kFoldThreads) k_batch_begin(const BatchParams bp,
                                                              long long max_steps,
                                                              int stop_on_done) {
  BatchCtl* b = bp.bctl;
  const BatchTab* tab = bp.tab;
  if (threadIdx.x < 32) batch_compact(bp);
  __syncthreads();
  const int nact = tab->nact;
  for (int a = threadIdx.x; a < nact; a += blockDim.x) batch_next<T>(&bp.scen[tab->act[a]]);
  if (threadIdx.x == 0) {
    const long long s = b->step;
    b->step_stop = (max_steps > (long long)0x3FFFFFFFFFFFFFFFLL - s) ? 0x3FFFFFFFFFFFFFFFLL
                                                                     : s + max_steps;
    b->completed = 0;
    b->next_unit = 0u;
    b->stop_on_done = stop_on_done;
    const int done = nact == 0 || max_steps <= 0 || b->status != 0;
    b->done = done;
    b->last_stamp = global_ns();
    __threadfence();
    if (bp.use_cond) cudaGraphSetConditional(bp.cond, done ? 0u : 1u);
  }
}

// Sum of the per-strip volume/area partials of one grid in a fixed order
// (lane l takes strips l, l+32, ..., Neumaier-compensated; then the lanes in
// order), by one warp; every lane gets the result.
__device__ inline void warp_fold_partials(const double* part, int n, double& vol, double& area) {
  const int lane = threadIdx.x & 31;
  double s = 0.0, c = 0.0, a = 0.0;
  for (int k = lane; k < n; k += 32) {
    kahan_add(s, c, part[3 * k]);
    a += part[3 * k + 2];
  }
  double S = 0.0, C = 0.0, A = 0.0;
  for (int l = 0; l < 32; l++) {
    kahan_add(S, C, __shfl_sync(0xffffffffu, s, l));
    C += __shfl_sync(0xffffffffu, c, l);
    A += __shfl_sync(0xffffffffu, a, l);
  }
  vol = S + C;
  area = A;
}

// Folds one batch step (one block): see the section comment.
template <typename T>
__global__ void __launch_bounds__(kFoldThreads) k_batch_fold(const BatchParams bp) {
  __shared__ double s_vol[kMaxSlots], s_area[kMaxSlots];
  BatchCtl* b = bp.bctl;
  if (*(volatile int*)&b->done) return;  // the loop ended at an earlier step
  const BatchTab* tab = bp.tab;
  const int nact = tab->nact;
  const long long step_cells = tab->cells;  // read before any recompaction below
  const int step_units = tab->units;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int a = warp; a < nact; a += nwarps) {  // volume sums of the reporting scenarios
    const BatchScen* s = &bp.scen[tab->act[a]];
    if (s->p.mass_int > 0.0 && s->t + s->dt >= s->next_mass) {
      double v, ar;
      warp_fold_partials(s->p.partials, s->p.nsx * s->p.nsy, v, ar);
      if (lane == 0) {
        s_vol[a] = v;
        s_area[a] = ar;
      }
    }
  }
  __syncthreads();
  int done = 0;
  for (int a = threadIdx.x; a < nact; a += blockDim.x) {
    BatchScen* s = &bp.scen[tab->act[a]];
    const bool mass = s->p.mass_int > 0.0 && s->t + s->dt >= s->next_mass;
    if (fold_step(s->p, s->p.ctl, s->t, s->dt, s->parity, mass, mass ? s_vol[a] : 0.0,
                  mass ? s_area[a] : 0.0))
      done++;
    else
      batch_next<T>(s);
  }
  const int ndone = __syncthreads_count(done);
  if (ndone > 0) {  // the active list changes only when a scenario finishes
    __threadfence();
    if (threadIdx.x < 32) batch_compact(bp);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const long long step_new = b->step + 1;
    b->next_unit = 0u;  // the next step hands out its units afresh
    b->step = step_new;
    b->completed += ndone;
    const bool attn = bp.attention != nullptr && *bp.attention != 0;
    const bool stop = tab->nact == 0 || step_new >= b->step_stop ||
                      *(volatile int*)&b->status != 0 || (b->stop_on_done && b->completed > 0) ||
                      attn;
    b->done = stop;
    if (b->trace != nullptr) {
      const long long k = step_new - 1 - b->trace_base;
      const unsigned long long now = global_ns();
      if (k >= 0 && k < b->trace_cap) {
        unsigned long long* r = b->trace + 4 * k;
        r[0] = b->last_stamp;
        r[1] = now;
        r[2] = (unsigned long long)step_cells;
        r[3] = (unsigned long long)step_units;
      }
      b->last_stamp = now;
    }
    __threadfence();
    if (bp.use_cond) cudaGraphSetConditional(bp.cond, stop ? 0u : 1u);
  }
}

template <typename T, int WY, int MINB>
__global__ void __launch_bounds__(32 * WY, MINB) k_batch_step(const BatchParams bp) {
  __shared__ __align__(128) unsigned char s_ring[WY][kStages][4][kRowBytes];
  __shared__ __align__(8) uint64_t s_bar[WY][kStages + 1];  // the ring's, then the records'
  __shared__ BatchScen s_rec[WY][2];
  if (*(volatile int*)&bp.bctl->done) return;
  const BatchTab* tab = bp.tab;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  uint64_t* bar = s_bar[warp];
  uint64_t* rbar = &s_bar[warp][kStages];
  if (lane == 0) {
    for (int s = 0; s <= kStages; s++) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncwarp();
  RingPos pos{0u};
  uint32_t rphase = 0;  // completed record fetches, mod 2
  const int units = tab->units;
  const int nact = tab->nact;
  const int W = gridDim.x * WY;
  // Active-scenario index of unit u, from the index `a` of an earlier unit
  // (u0 is increasing: count the entries past `a` that are <= u).
  auto scen_of = [&](int a, int u) {
    for (;;) {
      const int idx = a + 1 + lane;
      const bool le = idx < nact && tab->u0[idx] <= u;
      const unsigned m = __ballot_sync(0xffffffffu, le);
      a += __popc(m);
      if (m != 0xffffffffu) return a;
    }
  };
  // One bulk copy of a slot's record into buffer `b` (the warp has finished
  // reading that buffer: every lane has passed a __syncwarp since).
  auto fetch = [&](int slot, int b) {
    if (lane == 0) {
      mbar_expect_tx(rbar, (uint32_t)sizeof(BatchScen));
      fence_proxy_async();
      bulk_g2s(&s_rec[warp][b], &bp.scen[slot], (uint32_t)sizeof(BatchScen), rbar);
    }
  };
  auto fetched = [&]() {
    const bool ok = mbar_wait_warp(rbar, rphase);
    rphase ^= 1u;
    return ok;
  };
  int u = blockIdx.x * WY + warp;
  if (u >= units) return;
  int a = scen_of(0, u);
  int slot = tab->act[a];
  int buf = 0;
  fetch(slot, buf);
  bool ok = fetched();
  if (!ok) mbar_wait_warp(rbar, rphase ^ 1u);  // drain the copy before leaving
  while (ok) {
    // The next unit's scenario; its record is fetched while this unit runs.
#if AF_BATCH_DYNAMIC
    // After the first round a warp takes the next unfinished unit from the
    // step's counter (fetched one unit ahead, so the record prefetch still
    // overlaps): warps that finish early take more, none idles while units
    // remain.  Units keep their order, so warps running at once still read
    // neighbouring strips of the same rows.
    int un = 0;
    if (lane == 0) un = W + (int)atomicAdd(&bp.bctl->next_unit, 1u);
    un = __shfl_sync(0xffffffffu, un, 0);
#else
    const int un = u + W;
#endif
    const int an = un < units ? scen_of(a, un) : a;
    const int slot_n = un < units ? tab->act[an] : -1;
    const bool refetch = slot_n >= 0 && slot_n != slot;
    __syncwarp();
    if (refetch) fetch(slot_n, buf ^ 1);
    const BatchScen& rec = s_rec[warp][buf];
    const StepParams& p = rec.p;
    const StepScal<T>& sc = *reinterpret_cast<const StepScal<T>*>(rec.scal);
    const int k = u - tab->u0[a];
    LaneAcc<T> acc{T(-FLT_MAX), 0.0, 0.0};
    ok = run_strip<T, true>(p, sc, k % p.nsx, k / p.nsx, s_ring[warp], bar, pos, acc);
    double m = acc.any_cell() ? (double)acc.m_cell : -DBL_MAX;
    m = warp_maxd(m);
    double v = 0.0, ar = 0.0;
    if (sc.mass) {
      v = warp_sum(acc.v);
      ar = warp_sum(acc.a);
    }
    if (lane == 0) {
      if (m > -DBL_MAX) atomicMax(&p.ctl->hmax_acc, ord_encode(m));
      if (sc.mass) {
        p.partials[3 * k] = v;
        p.partials[3 * k + 1] = 0.0;
        p.partials[3 * k + 2] = ar;
      }
    }
    if (refetch) {
      // Waited for even after a failure: no copy may be in flight at exit.
      if (!fetched()) {
        mbar_wait_warp(rbar, rphase ^ 1u);
        ok = false;
      }
      buf ^= 1;
    }
    if (slot_n < 0) break;
    u = un;
    a = an;
    slot = slot_n;
  }
  // A wait timed out: this step's state is incomplete, so stop the batch.
  if (!ok && lane == 0) atomicExch(&bp.bctl->status, 1);
}

// Whether a single grid's FP64 step takes the kernel that evaluates each wet
// face out of line (k_step<double, ..., true>): on grids of more than 2^18
// and at most 2^25 cells (see face_q64).  AF_SIM_FACE_CALL=0/1 forces the
// choice (for measurements).
constexpr long long kFaceCallMinCells = (1LL << 18) + 1;
constexpr long long kFaceCallMaxCells = 1LL << 25;
inline bool face_call_for(bool f64, long long cells) {
  if (!f64) return false;
  if (const char* v = getenv("AF_SIM_FACE_CALL")) return v[0] == '1';
  return cells >= kFaceCallMinCells && cells <= kFaceCallMaxCells;
}
// Whether a single grid's step reads its rows with one tiled copy (TMA) per
// row instead of four bulk copies: FP32 grids of at most kTmaMaxCellsF32
// cells, FP64 grids of at most kTmaMaxCellsF64.  The tiled copies take fewer
// instructions but read a few per cent more DRAM bytes, so they pay where the
// step is bound by issue or latency and lose where it is bound by bandwidth.
// Measured, ms per FP32 step with tiled against bulk copies: 3072^2 0.0835 /
// 0.0868, 4096^2 0.1226 / 0.1273, 4608^2 0.1484 / 0.1507; 5120^2 0.1801 /
// 0.1734, 5792^2 0.2262 / 0.2140, 8192^2 0.432 / 0.369.  FP64, wet grids:
// 3-5 % faster at every size from 1024^2 to 16384^2 (8192^2 2.12 against
// 2.21 ms), but 6 % slower on the mostly dry 16384^2 start of the ponds
// configuration, where the FP64 step is bandwidth-bound too.
// AF_SIM_TMA=0/1 forces the choice.
constexpr long long kTmaMaxCellsF32 = 4700LL * 4700;
constexpr long long kTmaMaxCellsF64 = 1LL << 26;
inline bool tma_for(bool f64, long long cells) {
  if (const char* v = getenv("AF_SIM_TMA")) return v[0] == '1';
  return cells <= (f64 ? kTmaMaxCellsF64 : kTmaMaxCellsF32);
}

// The tensor map of a grid's field planes: 8 planes (H0, DEM, Qx0, Qy0, H1,
// DEM, Qx1, Qy1) `plane_bytes` apart from `origin` (the first plane's cell
// (0, 0)), rows P elements apart; x covers columns 0..nx (Qx's east face
// included), y rows 0..ny (Qy's last included), z the planes; a box is one
// 512-byte row window of 4 planes.  AF_ECUDA if the driver refuses it.
inline int encode_field_planes(CUtensorMap* out, void* origin, int esize, int nx, int ny, int P,
                               size_t plane_bytes) {
  using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return AF_ECUDA;
    encode = reinterpret_cast<EncodeFn>(fn);
  }
  const cuuint64_t dims[3] = {(cuuint64_t)nx + 1, (cuuint64_t)ny + 1, 8};
  const cuuint64_t strides[2] = {(cuuint64_t)P * esize, (cuuint64_t)plane_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)(kRowBytes / esize), 1, 4};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode(
      out, esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
      origin, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? AF_OK : AF_ECUDA;
}

// Kernel entry points of the two precisions (defined in af_step_f64.cu and
// af_step_f32.cu, which are compiled with different floating-point flags).
// Launch variants: (warps per block, minimum resident blocks per SM).
struct StepVariant {
  int wy, minb;
};
constexpr int kStepVariants = 5;
constexpr StepVariant kStepVariant[kStepVariants] = {{1, 16}, {1, 12}, {1, 20}, {4, 4}, {2, 8}};
const void* step_kernel_f64(int variant, bool face_call = false, bool tma = true);
const void* step_kernel_f32(int variant, bool tma = true);
const void* batch_kernel_f64(int variant);
const void* batch_kernel_f32(int variant);
// Begin and fold kernels of the batch loop (one block of kFoldThreads),
// compiled beside the step kernels of the same precision.
const void* batch_begin_f64();
const void* batch_begin_f32();
const void* batch_fold_f64();
const void* batch_fold_f32();

}  // namespace af
