// ref_driver.cpp -- runs the reference's own hot path on the CPU.
//
// TEST INFRASTRUCTURE ONLY (oracle).  This file is compiled together with the
// reference's unmodified src/kernels.cpp and src/io.cpp against the in-repo
// Kokkos-API shim (oracle/kokkos_shim) into oracle/_ref/libafref.so.  It is the
// checker that pins the C restatement (oracle/af_oracle.c) and the CUDA
// implementation; it is never part of the shipped library.
//
// Every statement inside afref_step() restates one line of the reference's
// time loop, src/main.cpp:227-288, in the same order, and calls the
// reference's own kernel functions (src/kernels.cpp) and interpolation
// (src/io.cpp:299-311, src/io.cpp:88-100).  Input parsing is the reference's
// own read_par/read_dem/read_bci/read_bdy/read_rain (src/io.cpp:9-296).
//
// Additions that have no counterpart in the reference:
//   * afref_set_h: an initial depth field (the reference hard-codes H = 0 at
//     src/main.cpp:156) so reservoir-style scenarios can be replayed;
//   * afref_run stops at a caller-given time or step count so the state can be
//     dumped at full precision (the reference only writes %.4f ASCII).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>
#include <fcntl.h>

#include "types.hpp"
#include "io.hpp"
#include "kernels.hpp"

namespace {

struct RefSim {
  Parameters par;
  int ncols = 0, nrows = 0;
  double xll = 0, yll = 0, cellsize = 0, nodata = 0;
  std::vector<PointBoundary> flow_bcs, other_bcs;
  bool west_free = false, east_free = false, north_free = false, south_free = false;
  RainfallData rainfall;
  // constants of src/main.cpp:115-124
  double dx = 0, dy = 0, dA = 0, FPn = 0, DepthThresh = 0, MaxHflow = 10.0, dhlin = 0.01,
         Qlimfact = 1.0, InitTstep = 0, cfl = 0, g = 9.81, theta = 1.0;
  RealView H, DEM, Qx, Qy, Qxold, Qyold, Vx, Vy;
  IntView ps_idx;
  RealView ps_flow;
  IntView bc_idx, bc_type;
  RealView bc_value;
  double t = 0.0;
  long step = 0;
  double last_dt = 0.0;
};

// Silences the reference's progress printf()s while a call runs.
struct Quiet {
  int saved = -1;
  explicit Quiet(bool on) {
    if (!on) return;
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) {
      dup2(devnull, 1);
      close(devnull);
    }
  }
  ~Quiet() {
    if (saved < 0) return;
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};

// One time step: src/main.cpp:227-288 in order.
void afref_step(RefSim& s) {
  const int ncols = s.ncols, nrows = s.nrows;
  double Tstep = s.InitTstep;                                       // main.cpp:228
  FloodplainQ_GPU(s.H, s.DEM, s.Qx, s.Qy, s.Qxold, s.Qyold, ncols, nrows, s.dx, s.dy, s.FPn,
                  s.DepthThresh, s.MaxHflow, s.dhlin, Tstep, s.Qlimfact, s.dA, s.cfl, s.g,
                  s.InitTstep, s.theta, s.nodata);                  // main.cpp:231
  BCs_GPU(s.Qx, s.Qy, s.H, s.DEM, ncols, nrows, s.dx, s.g, Tstep, s.nodata, s.west_free,
          s.east_free, s.north_free, s.south_free);                 // main.cpp:236
  const int num_flow_bcs = (int)s.flow_bcs.size();
  if (num_flow_bcs > 0) {                                           // main.cpp:245-262
    auto ps_flow_host = Kokkos::create_mirror_view(s.ps_flow);
    for (int k = 0; k < num_flow_bcs; k++) {
      double flow_val;
      if (s.flow_bcs[k].type == BC_QFIX) {
        flow_val = s.flow_bcs[k].value;
      } else {
        flow_val = interpolate_bc_value(s.flow_bcs[k], s.t);
      }
      ps_flow_host(k) = flow_val * s.dx * Tstep / s.dA;
    }
    Kokkos::deep_copy(s.ps_flow, ps_flow_host);
    RealView H = s.H;
    IntView ps_idx = s.ps_idx;
    RealView ps_flow = s.ps_flow;
    Kokkos::parallel_for("AddFlowBCs", num_flow_bcs, KOKKOS_LAMBDA(int k) {
      int idx = ps_idx(k);
      H(idx) += ps_flow(k);
      if (H(idx) < 0.0) H(idx) = 0.0;
    });
    Kokkos::fence();
  }
  if (s.rainfall.enabled) {                                         // main.cpp:265-268
    double rain_rate = interpolate_rain(s.rainfall, s.t);
    Rainfall_GPU(s.H, s.DEM, ncols, nrows, rain_rate, Tstep, s.nodata);
  }
  UpdateH_GPU(s.H, s.Qx, s.Qy, ncols, nrows, s.dA, Tstep);           // main.cpp:271
  const int num_other_bcs = (int)s.other_bcs.size();
  if (num_other_bcs > 0) {                                          // main.cpp:274-282
    auto bc_value_host = Kokkos::create_mirror_view(s.bc_value);
    for (int b = 0; b < num_other_bcs; b++) {
      if (s.other_bcs[b].type == BC_HVAR) {
        bc_value_host(b) = interpolate_bc_value(s.other_bcs[b], s.t);
      }
    }
    Kokkos::deep_copy(s.bc_value, bc_value_host);
    ApplyPointBCs_GPU(s.H, s.bc_idx, s.bc_type, s.bc_value, num_other_bcs, ncols, s.dx, s.dA,
                      Tstep);
  }
  UpdateQs_GPU(s.Qx, s.Qy, s.Qxold, s.Qyold, ncols, nrows, s.dx);   // main.cpp:285
  s.t += Tstep;                                                     // main.cpp:287
  s.step++;
  s.last_dt = Tstep;
}

}  // namespace

extern "C" {

// Loads a case through the reference's parsers and sets up the state exactly
// as src/main.cpp:24-194 does.  Returns nullptr on a parse failure.
void* afref_open(const char* parfile, int quiet) {
  Quiet q(quiet != 0);
  RefSim* s = new RefSim();
  if (!read_par(parfile, s->par)) { delete s; return nullptr; }
  std::vector<double> dem_data;
  if (!read_dem(s->par.dem_file.c_str(), s->ncols, s->nrows, s->xll, s->yll, s->cellsize,
                s->nodata, dem_data)) { delete s; return nullptr; }
  std::vector<PointBoundary> point_bcs;
  std::vector<LineBoundary> line_bcs;
  if (!read_bci(s->par.bci_file.c_str(), s->xll, s->yll, s->ncols, s->nrows, s->cellsize,
                point_bcs, line_bcs)) { delete s; return nullptr; }
  if (!read_bdy(s->par.bdy_file.c_str(), point_bcs)) { delete s; return nullptr; }
  for (const auto& lb : line_bcs) {                                 // main.cpp:62-70
    if (lb.type == BC_FREE) {
      if (lb.side == 'W') s->west_free = true;
      else if (lb.side == 'E') s->east_free = true;
      else if (lb.side == 'N') s->north_free = true;
      else if (lb.side == 'S') s->south_free = true;
    }
  }
  for (const auto& pb : point_bcs) {                                // main.cpp:77-85
    if (pb.type == BC_QVAR || pb.type == BC_QFIX) s->flow_bcs.push_back(pb);
    else s->other_bcs.push_back(pb);
  }
  if (!s->par.rain_file.empty()) read_rain(s->par.rain_file.c_str(), s->rainfall);

  s->dx = s->cellsize; s->dy = s->cellsize; s->dA = s->dx * s->dy;  // main.cpp:115-124
  s->FPn = s->par.fpn; s->DepthThresh = s->par.depth_thresh;
  s->InitTstep = s->par.init_tstep; s->cfl = s->par.cfl;

  const int n = s->ncols * s->nrows, f = (s->ncols + 1) * (s->nrows + 1);
  s->H = RealView("H", n);                                          // main.cpp:133-141
  s->DEM = RealView("DEM", n);
  s->Qx = RealView("Qx", f);
  s->Qy = RealView("Qy", f);
  s->Qxold = RealView("Qxold", f);
  s->Qyold = RealView("Qyold", f);
  s->Vx = RealView("Vx", n);
  s->Vy = RealView("Vy", n);
  for (int i = 0; i < n; i++) s->DEM(i) = dem_data[i];

  const int nf = (int)s->flow_bcs.size();                           // main.cpp:167-194
  s->ps_idx = IntView("ps_idx", nf > 0 ? nf : 1);
  s->ps_flow = RealView("ps_flow", nf > 0 ? nf : 1);
  for (int k = 0; k < nf; k++) s->ps_idx(k) = s->flow_bcs[k].idx;
  const int no = (int)s->other_bcs.size();
  s->bc_idx = IntView("bc_idx", no > 0 ? no : 1);
  s->bc_type = IntView("bc_type", no > 0 ? no : 1);
  s->bc_value = RealView("bc_value", no > 0 ? no : 1);
  for (int b = 0; b < no; b++) {
    s->bc_idx(b) = s->other_bcs[b].idx;
    if (s->other_bcs[b].type == BC_FREE) s->bc_type(b) = 1;
    else if (s->other_bcs[b].type == BC_HFIX) s->bc_type(b) = 2;
    else if (s->other_bcs[b].type == BC_HVAR) s->bc_type(b) = 3;
    s->bc_value(b) = s->other_bcs[b].value;
  }
  return s;
}

void afref_close(void* h) { delete static_cast<RefSim*>(h); }

// Builds the same state afref_open would, from arrays instead of files (for
// grids whose ASCII DEM would be gigabytes).  Flow boundaries are QFIX (4) /
// QVAR (5) in file order, other boundaries FREE (1) / HFIX (2) / HVAR (3);
// hydrographs are CSR (off[k]..off[k+1]).  params: sim_time, cfl, fpn,
// depth_thresh, init_tstep, mass_int; flags: west, east, north, south FREE.
void* afref_create(int ncols, int nrows, double cellsize, double nodata, const double* params,
                   const int* flags, const double* dem, int n_flow, const int* flow_idx,
                   const int* flow_type, const double* flow_value, const int* flow_off,
                   const double* flow_times, const double* flow_vals, int n_other,
                   const int* other_idx, const int* other_type, const double* other_value,
                   const int* other_off, const double* other_times, const double* other_vals,
                   int n_rain, const double* rain_times, const double* rain_rates) {
  RefSim* s = new RefSim();
  s->ncols = ncols;
  s->nrows = nrows;
  s->cellsize = cellsize;
  s->nodata = nodata;
  s->par.sim_time = params[0];
  s->par.cfl = params[1];
  s->par.fpn = params[2];
  s->par.depth_thresh = params[3];
  s->par.init_tstep = params[4];
  s->par.mass_int = params[5];
  s->west_free = flags[0] != 0;
  s->east_free = flags[1] != 0;
  s->north_free = flags[2] != 0;
  s->south_free = flags[3] != 0;
  for (int k = 0; k < n_flow; k++) {
    PointBoundary pb;
    pb.idx = flow_idx[k];
    pb.x = pb.idx % ncols;
    pb.y = pb.idx / ncols;
    pb.type = flow_type[k] == 4 ? BC_QFIX : BC_QVAR;
    pb.value = flow_value[k];
    for (int e = flow_off[k]; e < flow_off[k + 1]; e++) {
      pb.times.push_back(flow_times[e]);
      pb.values.push_back(flow_vals[e]);
    }
    s->flow_bcs.push_back(pb);
  }
  for (int k = 0; k < n_other; k++) {
    PointBoundary pb;
    pb.idx = other_idx[k];
    pb.x = pb.idx % ncols;
    pb.y = pb.idx / ncols;
    pb.type = other_type[k] == 1 ? BC_FREE : other_type[k] == 2 ? BC_HFIX : BC_HVAR;
    pb.value = other_value[k];
    for (int e = other_off[k]; e < other_off[k + 1]; e++) {
      pb.times.push_back(other_times[e]);
      pb.values.push_back(other_vals[e]);
    }
    s->other_bcs.push_back(pb);
  }
  for (int k = 0; k < n_rain; k++) {
    s->rainfall.times.push_back(rain_times[k]);
    s->rainfall.rates.push_back(rain_rates[k]);
  }
  s->rainfall.enabled = n_rain > 0;

  s->dx = s->cellsize; s->dy = s->cellsize; s->dA = s->dx * s->dy;  // main.cpp:115-124
  s->FPn = s->par.fpn; s->DepthThresh = s->par.depth_thresh;
  s->InitTstep = s->par.init_tstep; s->cfl = s->par.cfl;
  const long n = (long)ncols * nrows, f = (long)(ncols + 1) * (nrows + 1);
  s->H = RealView("H", n);
  s->DEM = RealView("DEM", n);
  s->Qx = RealView("Qx", f);
  s->Qy = RealView("Qy", f);
  s->Qxold = RealView("Qxold", f);
  s->Qyold = RealView("Qyold", f);
  s->Vx = RealView("Vx", n);
  s->Vy = RealView("Vy", n);
  std::memcpy(s->DEM.data(), dem, sizeof(double) * n);
  const int nf = n_flow, no = n_other;
  s->ps_idx = IntView("ps_idx", nf > 0 ? nf : 1);
  s->ps_flow = RealView("ps_flow", nf > 0 ? nf : 1);
  for (int k = 0; k < nf; k++) s->ps_idx(k) = s->flow_bcs[k].idx;
  s->bc_idx = IntView("bc_idx", no > 0 ? no : 1);
  s->bc_type = IntView("bc_type", no > 0 ? no : 1);
  s->bc_value = RealView("bc_value", no > 0 ? no : 1);
  for (int b = 0; b < no; b++) {
    s->bc_idx(b) = s->other_bcs[b].idx;
    s->bc_type(b) = other_type[b];
    s->bc_value(b) = s->other_bcs[b].value;
  }
  return s;
}

// Replaces H, Qx, Qy (reference layout) and t; Qold is re-formed with the
// reference's own UpdateQs_GPU, as after a completed step.
int afref_set_state(void* h, const double* H, const double* Qx, const double* Qy, double t) {
  RefSim* s = static_cast<RefSim*>(h);
  const long n = (long)s->ncols * s->nrows, f = (long)(s->ncols + 1) * (s->nrows + 1);
  if (H) std::memcpy(s->H.data(), H, sizeof(double) * n);
  if (Qx) std::memcpy(s->Qx.data(), Qx, sizeof(double) * f);
  if (Qy) std::memcpy(s->Qy.data(), Qy, sizeof(double) * f);
  UpdateQs_GPU(s->Qx, s->Qy, s->Qxold, s->Qyold, s->ncols, s->nrows, s->dx);
  s->t = t;
  return 0;
}

// dims[0..1] = ncols, nrows; geo[0..3] = xll, yll, cellsize, nodata;
// par[0..7] = sim_time, save_int, mass_int, init_tstep, cfl, fpn, depth_thresh, rain_enabled;
// flags[0..5] = west, east, north, south FREE, num_flow_bcs, num_other_bcs.
int afref_info(void* h, int* dims, double* geo, double* par, int* flags) {
  RefSim* s = static_cast<RefSim*>(h);
  dims[0] = s->ncols; dims[1] = s->nrows;
  geo[0] = s->xll; geo[1] = s->yll; geo[2] = s->cellsize; geo[3] = s->nodata;
  par[0] = s->par.sim_time; par[1] = s->par.save_int; par[2] = s->par.mass_int;
  par[3] = s->par.init_tstep; par[4] = s->par.cfl; par[5] = s->par.fpn;
  par[6] = s->par.depth_thresh; par[7] = s->rainfall.enabled ? 1.0 : 0.0;
  flags[0] = s->west_free; flags[1] = s->east_free; flags[2] = s->north_free;
  flags[3] = s->south_free; flags[4] = (int)s->flow_bcs.size();
  flags[5] = (int)s->other_bcs.size();
  return 0;
}

// Point boundaries after the reference's parse, in file order within each
// group.  idx/type/nser are filled for all flow BCs then all other BCs.
int afref_points(void* h, int* idx, int* type, double* value, int* nser) {
  RefSim* s = static_cast<RefSim*>(h);
  int k = 0;
  for (const auto* grp : {&s->flow_bcs, &s->other_bcs}) {
    for (const auto& pb : *grp) {
      idx[k] = pb.idx; type[k] = (int)pb.type; value[k] = pb.value;
      nser[k] = (int)pb.times.size();
      k++;
    }
  }
  return k;
}

int afref_set_h(void* h, const double* H0) {
  RefSim* s = static_cast<RefSim*>(h);
  const int n = s->ncols * s->nrows;
  for (int i = 0; i < n; i++) s->H(i) = H0[i];
  return 0;
}

// Steps while t < t_stop and fewer than max_steps steps were taken in this
// call.  dt_out (optional, max_steps entries) receives each step's Tstep.
long afref_run(void* h, double t_stop, long max_steps, double* dt_out) {
  RefSim* s = static_cast<RefSim*>(h);
  long k = 0;
  while (s->t < t_stop && k < max_steps) {
    afref_step(*s);
    if (dt_out) dt_out[k] = s->last_dt;
    k++;
  }
  return k;
}

double afref_time(void* h) { return static_cast<RefSim*>(h)->t; }
long afref_steps(void* h) { return static_cast<RefSim*>(h)->step; }

// Full-precision state in the reference's layout: H, Vx, Vy have ncols*nrows
// entries, Qx, Qy have (ncols+1)*(nrows+1).  Velocity comes from the
// reference's ComputeVelocity_GPU (src/kernels.cpp:293-351).
int afref_get(void* h, double* H, double* Qx, double* Qy, double* Vx, double* Vy) {
  RefSim* s = static_cast<RefSim*>(h);
  const int n = s->ncols * s->nrows, f = (s->ncols + 1) * (s->nrows + 1);
  if (Vx || Vy)
    ComputeVelocity_GPU(s->Vx, s->Vy, s->H, s->DEM, s->Qx, s->Qy, s->ncols, s->nrows, s->dx,
                        s->nodata);
  if (H) std::memcpy(H, s->H.data(), sizeof(double) * n);
  if (Qx) std::memcpy(Qx, s->Qx.data(), sizeof(double) * f);
  if (Qy) std::memcpy(Qy, s->Qy.data(), sizeof(double) * f);
  if (Vx) std::memcpy(Vx, s->Vx.data(), sizeof(double) * n);
  if (Vy) std::memcpy(Vy, s->Vy.data(), sizeof(double) * n);
  return 0;
}

// The mass report of src/main.cpp:292-298.
int afref_volume(void* h, double* vol, double* area) {
  RefSim* s = static_cast<RefSim*>(h);
  RealView H = s->H;
  const double dA = s->dA;
  double total_vol = 0.0, flood_area = 0.0;
  Kokkos::parallel_reduce("Vol", s->ncols * s->nrows,
      KOKKOS_LAMBDA(int i, double& v) { v += H(i) * dA; }, total_vol);
  Kokkos::parallel_reduce("Area", s->ncols * s->nrows,
      KOKKOS_LAMBDA(int i, double& a) { if (H(i) > 0.01) a += dA; }, flood_area);
  *vol = total_vol;
  *area = flood_area;
  return 0;
}

// Single-function entry points on caller arrays in the reference layout, so
// each reference kernel can be checked on its own.
void afref_floodplain_q(double* H, double* DEM, double* Qx, double* Qy, double* Qxold,
                        double* Qyold, int xsz, int ysz, double dx, double FPn,
                        double DepthThresh, double MaxHflow, double cfl, double g,
                        double InitTstep, double theta, double nodata, double* Tstep) {
  const int n = xsz * ysz, f = (xsz + 1) * (ysz + 1);
  RealView vH("H", n), vD("DEM", n), vQx("Qx", f), vQy("Qy", f), vQxo("Qxo", f), vQyo("Qyo", f);
  std::memcpy(vH.data(), H, sizeof(double) * n);
  std::memcpy(vD.data(), DEM, sizeof(double) * n);
  std::memcpy(vQx.data(), Qx, sizeof(double) * f);
  std::memcpy(vQy.data(), Qy, sizeof(double) * f);
  std::memcpy(vQxo.data(), Qxold, sizeof(double) * f);
  std::memcpy(vQyo.data(), Qyold, sizeof(double) * f);
  double ts = InitTstep;
  FloodplainQ_GPU(vH, vD, vQx, vQy, vQxo, vQyo, xsz, ysz, dx, dx, FPn, DepthThresh, MaxHflow,
                  0.01, ts, 1.0, dx * dx, cfl, g, InitTstep, theta, nodata);
  std::memcpy(Qx, vQx.data(), sizeof(double) * f);
  std::memcpy(Qy, vQy.data(), sizeof(double) * f);
  *Tstep = ts;
}

void afref_bcs(double* Qx, double* Qy, double* H, double* DEM, int xsz, int ysz, double dx,
               double g, double nodata, int wf, int ef, int nf, int sf) {
  const int n = xsz * ysz, f = (xsz + 1) * (ysz + 1);
  RealView vH("H", n), vD("DEM", n), vQx("Qx", f), vQy("Qy", f);
  std::memcpy(vH.data(), H, sizeof(double) * n);
  std::memcpy(vD.data(), DEM, sizeof(double) * n);
  std::memcpy(vQx.data(), Qx, sizeof(double) * f);
  std::memcpy(vQy.data(), Qy, sizeof(double) * f);
  BCs_GPU(vQx, vQy, vH, vD, xsz, ysz, dx, g, 0.0, nodata, wf != 0, ef != 0, nf != 0, sf != 0);
  std::memcpy(Qx, vQx.data(), sizeof(double) * f);
  std::memcpy(Qy, vQy.data(), sizeof(double) * f);
}

void afref_update_h(double* H, double* Qx, double* Qy, int xsz, int ysz, double dA,
                    double Tstep) {
  const int n = xsz * ysz, f = (xsz + 1) * (ysz + 1);
  RealView vH("H", n), vQx("Qx", f), vQy("Qy", f);
  std::memcpy(vH.data(), H, sizeof(double) * n);
  std::memcpy(vQx.data(), Qx, sizeof(double) * f);
  std::memcpy(vQy.data(), Qy, sizeof(double) * f);
  UpdateH_GPU(vH, vQx, vQy, xsz, ysz, dA, Tstep);
  std::memcpy(H, vH.data(), sizeof(double) * n);
}

void afref_velocity(double* Vx, double* Vy, double* H, double* DEM, double* Qx, double* Qy,
                    int xsz, int ysz, double dx, double nodata) {
  const int n = xsz * ysz, f = (xsz + 1) * (ysz + 1);
  RealView vVx("Vx", n), vVy("Vy", n), vH("H", n), vD("DEM", n), vQx("Qx", f), vQy("Qy", f);
  std::memcpy(vH.data(), H, sizeof(double) * n);
  std::memcpy(vD.data(), DEM, sizeof(double) * n);
  std::memcpy(vQx.data(), Qx, sizeof(double) * f);
  std::memcpy(vQy.data(), Qy, sizeof(double) * f);
  ComputeVelocity_GPU(vVx, vVy, vH, vD, vQx, vQy, xsz, ysz, dx, nodata);
  std::memcpy(Vx, vVx.data(), sizeof(double) * n);
  std::memcpy(Vy, vVy.data(), sizeof(double) * n);
}

void afref_rainfall(double* H, double* DEM, int xsz, int ysz, double rate, double Tstep,
                    double nodata) {
  const int n = xsz * ysz;
  RealView vH("H", n), vD("DEM", n);
  std::memcpy(vH.data(), H, sizeof(double) * n);
  std::memcpy(vD.data(), DEM, sizeof(double) * n);
  Rainfall_GPU(vH, vD, xsz, ysz, rate, Tstep, nodata);
  std::memcpy(H, vH.data(), sizeof(double) * n);
}

void afref_update_qs(double* Qx, double* Qy, double* Qxold, double* Qyold, int xsz, int ysz,
                     double dx) {
  const int f = (xsz + 1) * (ysz + 1);
  RealView vQx("Qx", f), vQy("Qy", f), vQxo("Qxo", f), vQyo("Qyo", f);
  std::memcpy(vQx.data(), Qx, sizeof(double) * f);
  std::memcpy(vQy.data(), Qy, sizeof(double) * f);
  UpdateQs_GPU(vQx, vQy, vQxo, vQyo, xsz, ysz, dx);
  std::memcpy(Qxold, vQxo.data(), sizeof(double) * f);
  std::memcpy(Qyold, vQyo.data(), sizeof(double) * f);
}

}  // extern "C"
