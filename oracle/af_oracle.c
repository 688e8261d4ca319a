/* af_oracle.c -- CPU restatement of AdaptFlood's local-inertial time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA implementation is
 * compared against; the shipped library never links or calls it.  It is
 * itself pinned against the reference's own sources compiled on the CPU
 * (oracle/ref_driver.cpp -> oracle/_ref/libafref.so) and against golden
 * vectors that build generated (tests/golden/).
 *
 * Every function restates one reference function with the same arithmetic in
 * the same order.  It must be compiled with -ffp-contract=off (no FMA
 * contraction) so each expression rounds exactly as written.
 *
 * Layout (the reference's, src/main.cpp:133-138):
 *   cells  c(i,j) = i + j*nx,            N = nx*ny entries (H, DEM, Vx, Vy)
 *   faces  f(i,j) = i + j*(nx+1),        F = (nx+1)*(ny+1) entries (Qx, Qy)
 *   Qx(i,j) is the west face of cell (i,j); Qy(i,j) the north face.
 *   Row j = 0 is the north edge (src/io.cpp:152-156).
 */
#include <math.h>
#include <float.h>
#include <stddef.h>
#include <string.h>
#include <stdlib.h>

#include "af_oracle.h"

static inline double getmax(double a, double b) { return (a > b) ? a : b; } /* types.hpp:14 */
static inline double getmin(double a, double b) { return (a < b) ? a : b; } /* types.hpp:15 */

/* src/kernels.cpp:29-33: Max-reduction of H over cells whose DEM is not
 * nodata; the Kokkos Max identity is the lowest double. */
double afo_find_hmax(const double* H, const double* DEM, long n, double nodata) {
  double m = -DBL_MAX;
  for (long i = 0; i < n; i++)
    if (DEM[i] != nodata && H[i] > m) m = H[i];
  return m;
}

/* src/kernels.cpp:36-43. */
double afo_timestep(double hmax, double depth_thresh, double cfl, double dx, double g,
                    double init_tstep) {
  if (hmax > depth_thresh) return cfl * dx / sqrt(g * hmax);
  return init_tstep;
}

/* src/kernels.cpp:46-93: interior x-faces, i in [0,nx-2], j in [0,ny-1],
 * writing face (i+1, j). */
void afo_qx(const double* H, const double* DEM, double* Qx, const double* Qxold,
            const double* Qyold, int xsz, int ysz, double dx, double FPn, double DepthThresh,
            double MaxHflow, double dt, double g, double theta, double nodata) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ysz; j++) {
    for (int i = 0; i < xsz - 1; i++) {
      int p0 = i + j * xsz, p1 = i + 1 + j * xsz;
      int pq0 = (i + 1) + j * (xsz + 1);
      double z0 = DEM[p0], z1 = DEM[p1];
      if (z0 == nodata || z1 == nodata) {
        Qx[pq0] = 0.0;
        continue;
      }
      double h0 = H[p0], h1 = H[p1];
      double fn = FPn;
      double y0 = z0 + h0, y1 = z1 + h1;
      double dh = y0 - y1;
      double Sf = -dh / dx;
      double hflow = getmax(y0, y1) - getmax(z0, z1);
      hflow = getmax(hflow, 0.0);
      hflow = getmin(hflow, MaxHflow);
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
        double denominator = 1.0 + g * dt * hflow * fn * fn * fabs(qvect) / pow(hflow, 10.0 / 3.0);
        Q = numerator / denominator * dx;
        if (Q * dh < 0.0) {
          numerator = q0 - (g * dt * hflow * Sf);
          Q = numerator / denominator * dx;
        }
      }
      Qx[pq0] = Q;
    }
  }
}

/* src/kernels.cpp:96-143: interior y-faces, i in [0,nx-1], j in [0,ny-2],
 * writing face (i, j+1).  Sf divides by dx (dx == dy in the reference). */
void afo_qy(const double* H, const double* DEM, double* Qy, const double* Qxold,
            const double* Qyold, int xsz, int ysz, double dx, double FPn, double DepthThresh,
            double MaxHflow, double dt, double g, double theta, double nodata) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ysz - 1; j++) {
    for (int i = 0; i < xsz; i++) {
      int p0 = i + j * xsz, p1 = i + (j + 1) * xsz;
      int pq0 = i + (j + 1) * (xsz + 1);
      double z0 = DEM[p0], z1 = DEM[p1];
      if (z0 == nodata || z1 == nodata) {
        Qy[pq0] = 0.0;
        continue;
      }
      double h0 = H[p0], h1 = H[p1];
      double fn = FPn;
      double y0 = z0 + h0, y1 = z1 + h1;
      double dh = y0 - y1;
      double Sf = -dh / dx;
      double hflow = getmax(y0, y1) - getmax(z0, z1);
      hflow = getmax(hflow, 0.0);
      hflow = getmin(hflow, MaxHflow);
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
        double denominator = 1.0 + g * dt * hflow * fn * fn * fabs(qvect) / pow(hflow, 10.0 / 3.0);
        Q = numerator / denominator * dx;
        if (Q * dh < 0.0) {
          numerator = q0 - (g * dt * hflow * Sf);
          Q = numerator / denominator * dx;
        }
      }
      Qy[pq0] = Q;
    }
  }
}

/* src/kernels.cpp:149-256: edge faces.  A FREE side writes nrows (or ncols)
 * faces; a CLOSED side zeroes nrows+1 (or ncols+1) entries, the extra entry
 * being the corner slot of the (nx+1)*(ny+1) array. */
void afo_bcs(double* Qx, double* Qy, const double* H, const double* DEM, int xsz, int ysz,
             double dx, double g, double nodata, int west_free, int east_free, int north_free,
             int south_free) {
  if (west_free) { /* kernels.cpp:154-179 */
    for (int j = 0; j < ysz; j++) {
      int p0 = 0 + j * xsz;
      double h0 = H[p0];
      double z0 = DEM[p0];
      if (z0 == nodata || h0 < 0.001) {
        Qx[j * (xsz + 1)] = 0.0;
      } else {
        int p1 = 1 + j * xsz;
        double h1 = H[p1];
        double z1 = DEM[p1];
        double y0 = z0 + h0;
        double y1 = z1 + h1;
        if (y0 > z0) {
          double Sf = (y1 - y0) / dx;
          if (Sf < 0) {
            Qx[j * (xsz + 1)] = -h0 * sqrt(g * h0) * dx * 0.5;
          } else {
            Qx[j * (xsz + 1)] = 0.0;
          }
        } else {
          Qx[j * (xsz + 1)] = 0.0;
        }
      }
    }
  } else { /* kernels.cpp:181-183 */
    for (int j = 0; j < ysz + 1; j++) Qx[j * (xsz + 1)] = 0.0;
  }
  if (east_free) { /* kernels.cpp:187-202 */
    for (int j = 0; j < ysz; j++) {
      int p0 = (xsz - 1) + j * xsz;
      double h0 = H[p0];
      double z0 = DEM[p0];
      if (z0 == nodata || h0 < 0.001) {
        Qx[xsz + j * (xsz + 1)] = 0.0;
      } else if (h0 > 0.001) {
        Qx[xsz + j * (xsz + 1)] = h0 * sqrt(g * h0) * dx * 0.5;
      } else {
        Qx[xsz + j * (xsz + 1)] = 0.0;
      }
    }
  } else { /* kernels.cpp:204-206 */
    for (int j = 0; j < ysz + 1; j++) Qx[xsz + j * (xsz + 1)] = 0.0;
  }
  if (north_free) { /* kernels.cpp:210-225 */
    for (int i = 0; i < xsz; i++) {
      double h0 = H[i];
      double z0 = DEM[i];
      if (z0 == nodata || h0 < 0.001) {
        Qy[i] = 0.0;
      } else if (h0 > 0.001) {
        Qy[i] = -h0 * sqrt(g * h0) * dx * 0.5;
      } else {
        Qy[i] = 0.0;
      }
    }
  } else { /* kernels.cpp:227-229 */
    for (int i = 0; i < xsz + 1; i++) Qy[i] = 0.0;
  }
  if (south_free) { /* kernels.cpp:233-248 */
    for (int i = 0; i < xsz; i++) {
      int p0 = i + (ysz - 1) * xsz;
      double h0 = H[p0];
      double z0 = DEM[p0];
      if (z0 == nodata || h0 < 0.001) {
        Qy[i + ysz * (xsz + 1)] = 0.0;
      } else if (h0 > 0.001) {
        Qy[i + ysz * (xsz + 1)] = h0 * sqrt(g * h0) * dx * 0.5;
      } else {
        Qy[i + ysz * (xsz + 1)] = 0.0;
      }
    }
  } else { /* kernels.cpp:250-252 */
    for (int i = 0; i < xsz + 1; i++) Qy[i + ysz * (xsz + 1)] = 0.0;
  }
}

/* src/main.cpp:253: the per-step source depth of one flow BC. */
double afo_source_depth(double flow_val, double dx, double Tstep, double dA) {
  return flow_val * dx * Tstep / dA;
}

/* src/main.cpp:256-260, applied in file order (duplicates accumulate). */
void afo_add_flow(double* H, const int* idx, const double* ps_flow, int n) {
  for (int s = 0; s < n; s++) {
    int c = idx[s];
    H[c] += ps_flow[s];
    if (H[c] < 0.0) H[c] = 0.0;
  }
}

/* src/kernels.cpp:354-367. */
void afo_rainfall(double* H, const double* DEM, long n, double rain_rate, double Tstep,
                  double nodata) {
  if (rain_rate <= 0.0) return;
  double rain_depth = rain_rate * Tstep;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    if (DEM[i] != nodata) {
      H[i] += rain_depth;
      if (H[i] < 0.0) H[i] = 0.0;
    }
  }
}

/* src/kernels.cpp:280-290. */
void afo_update_h(double* H, const double* Qx, const double* Qy, int xsz, int ysz, double dA,
                  double Tstep) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ysz; j++) {
    for (int i = 0; i < xsz; i++) {
      int idx = i + j * xsz;
      double Qx_in = Qx[i + j * (xsz + 1)], Qx_out = Qx[(i + 1) + j * (xsz + 1)];
      double Qy_in = Qy[i + j * (xsz + 1)], Qy_out = Qy[i + (j + 1) * (xsz + 1)];
      H[idx] += Tstep * (Qx_in - Qx_out + Qy_in - Qy_out) / dA;
      if (H[idx] < 0.0) H[idx] = 0.0;
    }
  }
}

/* src/kernels.cpp:259-277, in file order (a later BC on the same cell wins). */
void afo_point_bcs(double* H, const int* idx, const int* type, const double* value, int n) {
  for (int b = 0; b < n; b++) {
    if (type[b] == 1) H[idx[b]] = 0.0;
    else if (type[b] == 2 || type[b] == 3) H[idx[b]] = value[b];
  }
}

/* src/kernels.cpp:6-19 over all (nx+1)*(ny+1) entries. */
void afo_update_qs(const double* Qx, const double* Qy, double* Qxold, double* Qyold, int xsz,
                   int ysz, double dx) {
  double dxinv = 1.0 / dx;
  long f = (long)(xsz + 1) * (ysz + 1);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < f; k++) {
    Qxold[k] = Qx[k] * dxinv;
    Qyold[k] = Qy[k] * dxinv;
  }
}

/* src/kernels.cpp:293-351. */
void afo_velocity(double* Vx, double* Vy, const double* H, const double* DEM, const double* Qx,
                  const double* Qy, int xsz, int ysz, double dx, double nodata) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ysz; j++) {
    for (int i = 0; i < xsz; i++) {
      int idx = i + j * xsz;
      double z = DEM[idx], h = H[idx];
      if (z == nodata || h < 0.001) {
        Vx[idx] = 0.0;
        Vy[idx] = 0.0;
        continue;
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
  }
}

/* src/main.cpp:293-298 (serial order; the reference's order is backend
 * dependent, so sums are compared with a tolerance). */
void afo_volume_area(const double* H, long n, double dA, double* vol, double* area) {
  double v = 0.0, a = 0.0;
  for (long i = 0; i < n; i++) {
    v += H[i] * dA;
    if (H[i] > 0.01) a += dA;
  }
  *vol = v;
  *area = a;
}

/* src/io.cpp:299-311 (interpolate_bc_value) and src/io.cpp:88-100
 * (interpolate_rain): linear scan; n == 0 returns the fixed value. */
double afo_interp(const double* times, const double* values, int n, double fixed, double t) {
  if (n == 0) return fixed;
  if (t <= times[0]) return values[0];
  if (t >= times[n - 1]) return values[n - 1];
  for (int i = 0; i < n - 1; i++) {
    if (t >= times[i] && t < times[i + 1]) {
      double ratio = (t - times[i]) / (times[i + 1] - times[i]);
      return values[i] + ratio * (values[i + 1] - values[i]);
    }
  }
  return values[n - 1];
}

/* ---------------- whole-step driver: src/main.cpp:227-288 ---------------- */

struct afo_sim {
  afo_case c;
  long n, f;
  double *H, *DEM, *Qx, *Qy, *Qxold, *Qyold, *ps_flow, *bc_value;
  double t;
  long step;
};

afo_sim* afo_create(const afo_case* c, const double* dem, const double* h0) {
  afo_sim* s = (afo_sim*)calloc(1, sizeof(afo_sim));
  if (!s) return NULL;
  s->c = *c;
  s->n = (long)c->nx * c->ny;
  s->f = (long)(c->nx + 1) * (c->ny + 1);
  s->H = (double*)calloc(s->n > 0 ? s->n : 1, sizeof(double));
  s->DEM = (double*)calloc(s->n > 0 ? s->n : 1, sizeof(double));
  s->Qx = (double*)calloc(s->f, sizeof(double));
  s->Qy = (double*)calloc(s->f, sizeof(double));
  s->Qxold = (double*)calloc(s->f, sizeof(double));
  s->Qyold = (double*)calloc(s->f, sizeof(double));
  s->ps_flow = (double*)calloc(c->n_flow > 0 ? c->n_flow : 1, sizeof(double));
  s->bc_value = (double*)calloc(c->n_other > 0 ? c->n_other : 1, sizeof(double));
  memcpy(s->DEM, dem, sizeof(double) * s->n);
  if (h0) memcpy(s->H, h0, sizeof(double) * s->n);
  for (int b = 0; b < c->n_other; b++) s->bc_value[b] = c->other_value[b];
  return s;
}

void afo_destroy(afo_sim* s) {
  if (!s) return;
  free(s->H); free(s->DEM); free(s->Qx); free(s->Qy); free(s->Qxold); free(s->Qyold);
  free(s->ps_flow); free(s->bc_value);
  free(s);
}

double afo_step(afo_sim* s) {
  const afo_case* c = &s->c;
  const int nx = c->nx, ny = c->ny;
  const double dx = c->dx, dA = dx * dx;
  /* main.cpp:231 -> kernels.cpp:22-146 */
  double hmax = afo_find_hmax(s->H, s->DEM, s->n, c->nodata);
  double Tstep = afo_timestep(hmax, c->depth_thresh, c->cfl, dx, c->g, c->init_tstep);
  afo_qx(s->H, s->DEM, s->Qx, s->Qxold, s->Qyold, nx, ny, dx, c->fpn, c->depth_thresh,
         c->max_hflow, Tstep, c->g, c->theta, c->nodata);
  afo_qy(s->H, s->DEM, s->Qy, s->Qxold, s->Qyold, nx, ny, dx, c->fpn, c->depth_thresh,
         c->max_hflow, Tstep, c->g, c->theta, c->nodata);
  /* main.cpp:236 */
  afo_bcs(s->Qx, s->Qy, s->H, s->DEM, nx, ny, dx, c->g, c->nodata, c->west_free, c->east_free,
          c->north_free, c->south_free);
  /* main.cpp:245-262 */
  if (c->n_flow > 0) {
    for (int k = 0; k < c->n_flow; k++) {
      double v;
      if (c->flow_type[k] == AFO_QFIX) {
        v = c->flow_value[k];
      } else {
        int o = c->flow_off[k];
        v = afo_interp(c->flow_times + o, c->flow_vals + o, c->flow_off[k + 1] - o,
                       c->flow_value[k], s->t);
      }
      s->ps_flow[k] = afo_source_depth(v, dx, Tstep, dA);
    }
    afo_add_flow(s->H, c->flow_idx, s->ps_flow, c->n_flow);
  }
  /* main.cpp:265-268 */
  if (c->n_rain > 0) {
    double rate = afo_interp(c->rain_times, c->rain_rates, c->n_rain, 0.0, s->t);
    afo_rainfall(s->H, s->DEM, s->n, rate, Tstep, c->nodata);
  }
  /* main.cpp:271 */
  afo_update_h(s->H, s->Qx, s->Qy, nx, ny, dA, Tstep);
  /* main.cpp:274-282 */
  if (c->n_other > 0) {
    for (int b = 0; b < c->n_other; b++) {
      if (c->other_type[b] == 3) {
        int o = c->other_off[b];
        s->bc_value[b] = afo_interp(c->other_times + o, c->other_vals + o,
                                    c->other_off[b + 1] - o, c->other_value[b], s->t);
      }
    }
    afo_point_bcs(s->H, c->other_idx, c->other_type, s->bc_value, c->n_other);
  }
  /* main.cpp:285 */
  afo_update_qs(s->Qx, s->Qy, s->Qxold, s->Qyold, nx, ny, dx);
  /* main.cpp:287-288 */
  s->t += Tstep;
  s->step++;
  return Tstep;
}

long afo_run(afo_sim* s, double t_stop, long max_steps, double* dt_out) {
  long k = 0;
  while (s->t < t_stop && k < max_steps) {
    double dt = afo_step(s);
    if (dt_out) dt_out[k] = dt;
    k++;
  }
  return k;
}

double afo_time(const afo_sim* s) { return s->t; }
long afo_steps(const afo_sim* s) { return s->step; }

void afo_get(const afo_sim* s, double* H, double* Qx, double* Qy, double* Vx, double* Vy) {
  if (H) memcpy(H, s->H, sizeof(double) * s->n);
  if (Qx) memcpy(Qx, s->Qx, sizeof(double) * s->f);
  if (Qy) memcpy(Qy, s->Qy, sizeof(double) * s->f);
  if (Vx && Vy)
    afo_velocity(Vx, Vy, s->H, s->DEM, s->Qx, s->Qy, s->c.nx, s->c.ny, s->c.dx, s->c.nodata);
}

void afo_set_state(afo_sim* s, const double* H, const double* Qx, const double* Qy, double t) {
  if (H) memcpy(s->H, H, sizeof(double) * s->n);
  if (Qx) {
    memcpy(s->Qx, Qx, sizeof(double) * s->f);
  }
  if (Qy) {
    memcpy(s->Qy, Qy, sizeof(double) * s->f);
  }
  afo_update_qs(s->Qx, s->Qy, s->Qxold, s->Qyold, s->c.nx, s->c.ny, s->c.dx);
  s->t = t;
}
