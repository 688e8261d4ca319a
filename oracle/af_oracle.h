/* af_oracle.h -- CPU restatement of AdaptFlood's time step (test infrastructure;
 * see af_oracle.c).  Not part of the shipped library. */
#ifndef AF_ORACLE_H
#define AF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { AFO_FREE = 1, AFO_HFIX = 2, AFO_HVAR = 3, AFO_QFIX = 4, AFO_QVAR = 5 };

/* One case after parsing: grid, parameters, and the forcing tables.  Flow
 * sources (QFIX/QVAR) and other point BCs (FREE/HFIX/HVAR, typed 1/2/3 as on
 * the device in src/main.cpp:187-189) each keep file order; hydrographs are
 * in CSR form (off[k]..off[k+1] into times/vals). */
typedef struct afo_case {
  int nx, ny;
  double dx, nodata, fpn, depth_thresh, cfl, init_tstep, g, max_hflow, theta;
  int west_free, east_free, north_free, south_free;
  int n_flow;
  const int* flow_idx;
  const int* flow_type;
  const double* flow_value;
  const int* flow_off;
  const double* flow_times;
  const double* flow_vals;
  int n_other;
  const int* other_idx;
  const int* other_type;
  const double* other_value;
  const int* other_off;
  const double* other_times;
  const double* other_vals;
  int n_rain;
  const double* rain_times;
  const double* rain_rates;
} afo_case;

typedef struct afo_sim afo_sim;

double afo_find_hmax(const double* H, const double* DEM, long n, double nodata);
double afo_timestep(double hmax, double depth_thresh, double cfl, double dx, double g,
                    double init_tstep);
void afo_qx(const double* H, const double* DEM, double* Qx, const double* Qxold,
            const double* Qyold, int xsz, int ysz, double dx, double FPn, double DepthThresh,
            double MaxHflow, double dt, double g, double theta, double nodata);
void afo_qy(const double* H, const double* DEM, double* Qy, const double* Qxold,
            const double* Qyold, int xsz, int ysz, double dx, double FPn, double DepthThresh,
            double MaxHflow, double dt, double g, double theta, double nodata);
void afo_bcs(double* Qx, double* Qy, const double* H, const double* DEM, int xsz, int ysz,
             double dx, double g, double nodata, int west_free, int east_free, int north_free,
             int south_free);
double afo_source_depth(double flow_val, double dx, double Tstep, double dA);
void afo_add_flow(double* H, const int* idx, const double* ps_flow, int n);
void afo_rainfall(double* H, const double* DEM, long n, double rain_rate, double Tstep,
                  double nodata);
void afo_update_h(double* H, const double* Qx, const double* Qy, int xsz, int ysz, double dA,
                  double Tstep);
void afo_point_bcs(double* H, const int* idx, const int* type, const double* value, int n);
void afo_update_qs(const double* Qx, const double* Qy, double* Qxold, double* Qyold, int xsz,
                   int ysz, double dx);
void afo_velocity(double* Vx, double* Vy, const double* H, const double* DEM, const double* Qx,
                  const double* Qy, int xsz, int ysz, double dx, double nodata);
void afo_volume_area(const double* H, long n, double dA, double* vol, double* area);
double afo_interp(const double* times, const double* values, int n, double fixed, double t);

afo_sim* afo_create(const afo_case* c, const double* dem, const double* h0);
void afo_destroy(afo_sim* s);
double afo_step(afo_sim* s);
long afo_run(afo_sim* s, double t_stop, long max_steps, double* dt_out);
double afo_time(const afo_sim* s);
long afo_steps(const afo_sim* s);
void afo_get(const afo_sim* s, double* H, double* Qx, double* Qy, double* Vx, double* Vy);
void afo_set_state(afo_sim* s, const double* H, const double* Qx, const double* Qy, double t);

#ifdef __cplusplus
}
#endif
#endif
