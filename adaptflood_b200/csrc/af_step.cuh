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

#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>

#include "af_common.cuh"

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
  unsigned int arrive;          // blocks finished in this step
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
  // special cells per strip (CSR over strip id = sy*nsx + sx, sorted by row, col)
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

__device__ inline void ld_vec(const double* p, double (&v)[2]) {
  double2 t = __ldg(reinterpret_cast<const double2*>(p));
  v[0] = t.x;
  v[1] = t.y;
}
__device__ inline void ld_vec(const float* p, float (&v)[4]) {
  float4 t = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = t.x;
  v[1] = t.y;
  v[2] = t.z;
  v[3] = t.w;
}
__device__ inline void st_vec(double* p, const double (&v)[2]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}
__device__ inline void st_vec(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// pow(hflow, 10/3): FP64 uses CUDA's pow (a few ulp from glibc's); FP32 uses
// exp2(10/3 * log2(h)) on the special-function unit.
__device__ inline double pow_10_3(double h) { return pow(h, 10.0 / 3.0); }
__device__ inline float pow_10_3(float h) { return exp2f((10.0f / 3.0f) * __log2f(h)); }

template <typename T>
struct Phys {
  T dx, fn, depth_thresh, max_hflow, nodata, gdt;  // gdt = g*dt
  T g;
};

// Interior face flux with theta == 1 (src/kernels.cpp:51-92 / :101-142).
// Cell 0 is west (x-face) or north (y-face) of the face; qa..qd are the
// four cross-direction Qold values in the reference's summation order.
template <typename T>
__device__ inline T face_flux(T z0, T h0, T z1, T h1, T q0, T qa, T qb, T qc, T qd,
                              const Phys<T>& ph) {
  if (z0 == ph.nodata || z1 == ph.nodata) return T(0);
  T y0 = z0 + h0, y1 = z1 + h1;
  T dh = y0 - y1;
  T Sf = -dh / ph.dx;
  T hflow = gmaxT(y0, y1) - gmaxT(z0, z1);
  hflow = gmaxT(hflow, T(0));
  hflow = gminT(hflow, ph.max_hflow);
  T Q = T(0);
  if (hflow > ph.depth_thresh) {
    T q_avg = (qa + qb + qc + qd) / T(4);
    T qvect = sqrt(q0 * q0 + q_avg * q_avg);
    // theta*q0 + 0.5*(1-theta)*(qup+qdown) with theta == 1 is q0 + 0.
    T numerator = (q0 + T(0)) - (ph.gdt * hflow * Sf);
    T denominator = T(1) + ph.gdt * hflow * ph.fn * ph.fn * fabs(qvect) / pow_10_3(hflow);
    Q = numerator / denominator * ph.dx;
    if (Q * dh < T(0)) {
      numerator = q0 - (ph.gdt * hflow * Sf);
      Q = numerator / denominator * ph.dx;
    }
  }
  return Q;
}

// FREE edges (src/kernels.cpp:154-248).  West also needs the cell east of
// the edge cell.
template <typename T>
__device__ inline T west_free(T h0, T z0, T h1, T z1, const Phys<T>& ph) {
  if (z0 == ph.nodata || h0 < T(0.001)) return T(0);
  T y0 = z0 + h0, y1 = z1 + h1;
  if (y0 > z0) {
    T Sf = (y1 - y0) / ph.dx;
    if (Sf < 0) return -h0 * sqrt(ph.g * h0) * ph.dx * T(0.5);
  }
  return T(0);
}
template <typename T>
__device__ inline T out_free(T h0, T z0, T sign, const Phys<T>& ph) {
  if (z0 == ph.nodata || h0 < T(0.001)) return T(0);
  if (h0 > T(0.001)) return sign * h0 * sqrt(ph.g * h0) * ph.dx * T(0.5);
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

template <typename T>
__device__ inline T apply_sources(T h, const SpecCell& e, const StepParams& p, double t, double dt) {
  for (int s = e.s0; s < e.s1; s++) {
    double v;
    if (p.src_type[s] == AF_BC_QFIX) {
      v = p.src_value[s];
    } else {
      int o = p.src_off[s];
      v = interp_series(p.src_times + o, p.src_vals + o, p.src_off[s + 1] - o, p.src_value[s], t,
                        p.src_sorted[s] != 0);
    }
    double ps = v * p.dx * dt / p.dA;  // src/main.cpp:253
    h = h + T(ps);
    if (h < T(0)) h = T(0);
  }
  return h;
}

template <typename T>
__device__ inline T bc_depth(int b, const StepParams& p, double t) {
  int ty = p.bc_type[b];
  if (ty == 1) return T(0);
  if (ty == 2) return T(p.bc_value[b]);
  int o = p.bc_off[b];
  return T(interp_series(p.bc_times + o, p.bc_vals + o, p.bc_off[b + 1] - o, p.bc_value[b], t,
                         p.bc_sorted[b] != 0));
}

template <typename T, int WX>
__global__ void __launch_bounds__(32 * WX) k_step(const StepParams p) {
  constexpr int N = Lanes<T>::N;
  constexpr int OWN = 30 * N;
  SimCtl* ctl = p.ctl;
  if (*(volatile int*)&ctl->done) return;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sx = blockIdx.x * WX + warp;
  const int sy = blockIdx.y;
  const int parity = ctl->parity;
  const double t = ctl->t;
  const double hmax_prev = ctl->hmax;
  // src/kernels.cpp:36-43
  const double dt = (hmax_prev > p.depth_thresh) ? p.cfl * p.dx / sqrt(p.g * hmax_prev)
                                                 : p.init_tstep;
  const bool mass = p.mass_int > 0.0 && (t + dt >= ctl->next_mass);
  const double rate = ctl->rain_rate;
  const bool rain_on = rate > 0.0;  // src/kernels.cpp:356
  const T rain_depth = T(rate * dt);
  const T dtT = T(dt), dAT = T(p.dA), dxinvT = T(p.dxinv);

  Phys<T> ph;
  ph.dx = T(p.dx);
  ph.fn = T(p.fpn);
  ph.depth_thresh = T(p.depth_thresh);
  ph.max_hflow = T(p.max_hflow);
  ph.nodata = T(p.nodata);
  ph.g = T(p.g);
  ph.gdt = T(p.g * dt);  // (g*dt) rounded once, as the reference's left-to-right product does

  double m_loc = -DBL_MAX, v_loc = 0.0, a_loc = 0.0;

  if (sx < p.nsx) {
    const int nx = p.nx, ny = p.ny, P = p.P;
    const T* __restrict__ H = static_cast<const T*>(p.H[parity]);
    T* __restrict__ Hn = static_cast<T*>(p.H[parity ^ 1]);
    const T* __restrict__ Qx = static_cast<const T*>(p.Qx[parity]);
    T* __restrict__ Qxn = static_cast<T*>(p.Qx[parity ^ 1]);
    const T* __restrict__ Qy = static_cast<const T*>(p.Qy[parity]);
    T* __restrict__ Qyn = static_cast<T*>(p.Qy[parity ^ 1]);
    const T* __restrict__ Z = static_cast<const T*>(p.DEM);

    const int x0 = sx * OWN;
    const int cb = x0 - N + lane * N;  // first column of this lane
    const bool own = lane >= 1 && lane <= 30;
    const int j0 = sy * p.R;
    const int j1 = min(j0 + p.R, ny);
    const int strip = sy * p.nsx + sx;
    int sp = p.spec_off[strip];
    const int sp_end = p.spec_off[strip + 1];

    T h[N], z[N], qxo[N], qyo[N], qyn[N];
    {
      const long long r = (long long)j0 * P + cb;
      ld_vec(H + r, h);
      ld_vec(Z + r, z);
      ld_vec(Qx + r, qxo);
      ld_vec(Qy + r, qyo);
#pragma unroll
      for (int k = 0; k < N; k++) {
        qxo[k] = qxo[k] * dxinvT;
        qyo[k] = qyo[k] * dxinvT;
      }
    }
    // North faces of row j0.
    if (j0 == 0) {
#pragma unroll
      for (int k = 0; k < N; k++) qyn[k] = p.nf ? out_free(h[k], z[k], T(-1), ph) : T(0);
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
      T hp[N], zp[N], qxp[N];
      const long long r = (long long)(j0 - 1) * P + cb;
      ld_vec(H + r, hp);
      ld_vec(Z + r, zp);
      ld_vec(Qx + r, qxp);
#pragma unroll
      for (int k = 0; k < N; k++) qxp[k] = qxp[k] * dxinvT;
      T qxpR = __shfl_down_sync(0xffffffffu, qxp[0], 1);
      T qxoR = __shfl_down_sync(0xffffffffu, qxo[0], 1);
#pragma unroll
      for (int k = 0; k < N; k++) {
        T qb = (k < N - 1) ? qxp[k + 1] : qxpR;
        T qd = (k < N - 1) ? qxo[k + 1] : qxoR;
        qyn[k] = face_flux(zp[k], hp[k], z[k], h[k], qyo[k], qxp[k], qb, qxo[k], qd, ph);
      }
    }

    for (int j = j0; j < j1; j++) {
      const bool has_next = (j + 1 < ny);
      T hN[N], zN[N], qxoN[N], qyoN[N];
      {
        const long long r = (long long)(j + 1) * P + cb;
        ld_vec(Qy + r, qyoN);
        if (has_next) {
          ld_vec(H + r, hN);
          ld_vec(Z + r, zN);
          ld_vec(Qx + r, qxoN);
        } else {
#pragma unroll
          for (int k = 0; k < N; k++) hN[k] = zN[k] = qxoN[k] = T(0);
        }
#pragma unroll
        for (int k = 0; k < N; k++) {
          qyoN[k] = qyoN[k] * dxinvT;
          qxoN[k] = qxoN[k] * dxinvT;
        }
      }
      // Neighbours across lanes.
      const T hL = __shfl_up_sync(0xffffffffu, h[N - 1], 1);
      const T zL = __shfl_up_sync(0xffffffffu, z[N - 1], 1);
      const T qyoL = __shfl_up_sync(0xffffffffu, qyo[N - 1], 1);
      const T qyoNL = __shfl_up_sync(0xffffffffu, qyoN[N - 1], 1);
      const T qxoR = __shfl_down_sync(0xffffffffu, qxo[0], 1);
      const T qxoNR = __shfl_down_sync(0xffffffffu, qxoN[0], 1);

      // West face of every cell (face c between cells c-1 and c).
      T qw[N];
#pragma unroll
      for (int k = 0; k < N; k++) {
        const int c = cb + k;
        if (c == 0) {
          qw[k] = p.wf ? west_free(h[0], z[0], h[1], z[1], ph) : T(0);
        } else if (c < nx) {
          T hl = k ? h[k - 1] : hL;
          T zl = k ? z[k - 1] : zL;
          T qa = k ? qyo[k - 1] : qyoL;
          T qc = k ? qyoN[k - 1] : qyoNL;
          qw[k] = face_flux(zl, hl, z[k], h[k], qxo[k], qa, qyo[k], qc, qyoN[k], ph);
        } else {
          qw[k] = T(0);
        }
      }
      const T qwR = __shfl_down_sync(0xffffffffu, qw[0], 1);
      // South face of every cell (face row j+1).
      T qs[N];
#pragma unroll
      for (int k = 0; k < N; k++) {
        if (!has_next) {
          qs[k] = p.sf ? out_free(h[k], z[k], T(1), ph) : T(0);
        } else {
          T qb = (k < N - 1) ? qxo[k + 1] : qxoR;
          T qd = (k < N - 1) ? qxoN[k + 1] : qxoNR;
          qs[k] = face_flux(z[k], h[k], zN[k], hN[k], qyoN[k], qxo[k], qb, qxoN[k], qd, ph);
        }
      }
      // Depth update of the owned cells.
      T hn[N];
#pragma unroll
      for (int k = 0; k < N; k++) hn[k] = h[k];
      const int sp_row = sp;
      // Point sources (src/main.cpp:245-262), before rain and the update.
      while (sp < sp_end && p.spec[sp].row == j) {
        const SpecCell e = p.spec[sp];
        if (own) {
#pragma unroll
          for (int k = 0; k < N; k++)
            if (cb + k == e.col) hn[k] = apply_sources(hn[k], e, p, t, dt);
        }
        sp++;
      }
      T qe_last = T(0);
#pragma unroll
      for (int k = 0; k < N; k++) {
        const int c = cb + k;
        T qe;
        if (c == nx - 1) qe = p.ef ? out_free(h[k], z[k], T(1), ph) : T(0);
        else qe = (k < N - 1) ? qw[k + 1] : qwR;
        if (c == nx - 1) qe_last = qe;
        T v = hn[k];
        if (rain_on && z[k] != ph.nodata) {  // src/kernels.cpp:360-365
          v = v + rain_depth;
          if (v < T(0)) v = T(0);
        }
        v = v + dtT * (qw[k] - qe + qyn[k] - qs[k]) / dAT;  // src/kernels.cpp:286
        if (v < T(0)) v = T(0);
        hn[k] = v;
      }
      // Point depth BCs (src/kernels.cpp:259-277), after the update.
      for (int q = sp_row; q < sp; q++) {
        const SpecCell e = p.spec[q];
        if (own && e.bc >= 0) {
          const T v = bc_depth<T>(e.bc, p, t);
#pragma unroll
          for (int k = 0; k < N; k++)
            if (cb + k == e.col) hn[k] = v;
        }
      }
      if (own) {
        const long long r = (long long)j * P + cb;
        const long long rs = (long long)(j + 1) * P + cb;
        if (cb + N <= nx) {
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
        if (cb <= nx - 1 && nx - 1 < cb + N) Qxn[(long long)j * P + nx] = qe_last;
#pragma unroll
        for (int k = 0; k < N; k++) {
          if (cb + k < nx) {
            const double hv = (double)hn[k];
            if (z[k] != ph.nodata && hv > m_loc) m_loc = hv;
            if (mass) {
              v_loc += hv * p.dA;
              if (hv > 0.01) a_loc += p.dA;
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
  }

  // ----- block reductions: Hmax, and volume/area at mass-report steps -----
  __shared__ double s_m[WX], s_v[WX], s_a[WX];
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
    for (int w = 1; w < WX; w++) {
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
  __shared__ double r_v[32 * WX], r_c[32 * WX], r_a[32 * WX];
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
        p.mass_series[3 * k + 1] = r_v[0];
        p.mass_series[3 * k + 2] = r_a[0];
        ctl->mass_count = k + 1;
      }
      ctl->next_mass += p.mass_int;
    }
    ctl->rain_rate = p.n_rain > 0 ? interp_series(p.rain_times, p.rain_rates, p.n_rain, 0.0, t_new,
                                                  p.rain_sorted != 0)
                                  : 0.0;
    // A non-positive or non-finite dt (a diverged state) would stall time:
    // stop the loop and report it instead.
    const bool bad = !(dt > 0.0) || !(t_new < 1.0e300) || !(hmax == hmax);
    if (bad) ctl->status = 1;
    const int done = bad || !(t_new < ctl->t_stop) || step_new >= ctl->step_stop;
    ctl->done = done;
    ctl->arrive = 0u;
    __threadfence();
    if (p.use_cond) cudaGraphSetConditional(p.cond, done ? 0u : 1u);
  }
}

// Kernel entry points of the two precisions (defined in af_step_f64.cu and
// af_step_f32.cu, which are compiled with different floating-point flags).
const void* step_kernel_f64(int wx);
const void* step_kernel_f32(int wx);

}  // namespace af
